// C ABI of libscgpu.so (include/scg.h): the index handle, loaders, and the
// host orchestration of the batched search and the encoders.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <mutex>
#include <string>
#include <vector>

#include "index.h"

namespace scg {

static thread_local std::string g_err;

void set_error(const std::string &msg) { g_err = msg; }
std::string last_error_string() { return g_err; }
int fail(int code, const std::string &msg) {
    g_err = msg;
    return code;
}
int cuda_fail(cudaError_t e, const char *what) {
    g_err = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? SCG_ERR_OOM : SCG_ERR_CUDA;
}

}  // namespace scg

using namespace scg;

namespace scg {

int set_device(scg_index *h) {
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    return SCG_OK;
}

// A blocking host-to-device copy ordered before later work on stream s.  A
// plain cudaMemcpy runs on the legacy stream, which the index's non-blocking
// streams do not wait for, and from pageable memory it may return before its
// DMA has landed: a kernel launched next on s could read the buffer's tail
// before it arrives.
cudaError_t copy_in(void *dst, const void *src, size_t bytes, cudaStream_t s) {
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e;
}

bool read_file(const char *path, std::vector<unsigned char> &buf) {
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    if (!f) return false;
    std::streamsize n = f.tellg();
    if (n < 0) return false;
    f.seekg(0);
    buf.resize((size_t)n);
    return n == 0 || (bool)f.read((char *)buf.data(), n);
}

// Reads a .ctr_ file: float {k, m, dim} then k*dim floats
// (load_codebook, sc_utilities.h:897-980).
int read_ctr(const char *path, std::vector<float> &c, int &k, int &m, int &dim) {
    std::vector<unsigned char> b;
    if (!path || !read_file(path, b)) return fail(SCG_ERR_IO, std::string("cannot read codebook ") + (path ? path : "(null)"));
    if (b.size() < 12) return fail(SCG_ERR_IO, std::string("codebook too short: ") + path);
    float hdr[3];
    memcpy(hdr, b.data(), 12);
    k = (int)hdr[0];
    m = (int)hdr[1];
    dim = (int)hdr[2];
    if (k <= 0 || m <= 0 || dim <= 0 || dim % m != 0)
        return fail(SCG_ERR_IO, std::string("bad codebook header in ") + path);
    size_t need = (size_t)k * dim;
    if (b.size() < 12 + need * 4) return fail(SCG_ERR_IO, std::string("codebook truncated: ") + path);
    c.resize(need);
    memcpy(c.data(), b.data() + 12, need * 4);
    return SCG_OK;
}

int64_t ipow(int64_t b, int e) {
    int64_t r = 1;
    for (int i = 0; i < e; i++) r *= b;
    return r;
}

int check_ready(scg_index *h) {
    if (!h) return fail(SCG_ERR_ARG, "null index");
    if (!h->have_codebooks) return fail(SCG_ERR_STATE, "codebooks not loaded");
    if (!h->have_csr) return fail(SCG_ERR_STATE, "encoded data not loaded");
    if (!h->precomputed) return fail(SCG_ERR_STATE, "scg_precompute not called");
    return SCG_OK;
}

int check_params(scg_index *h, const scg_search_params *p, int nq) {
    if (!p) return fail(SCG_ERR_ARG, "null params");
    if (nq < 0) return fail(SCG_ERR_ARG, "nq < 0");
    if (p->R < 1 || p->R > 1024) return fail(SCG_ERR_ARG, "R must be in [1, 1024]");
    if (p->precision < SCG_FP32_EXACT || p->precision > SCG_FP16) return fail(SCG_ERR_ARG, "unknown precision");
    if (p->rerank < -1) return fail(SCG_ERR_ARG, "rerank must be -1, 0 or a shortlist length L");
    if (p->rerank > 0 && (p->rerank < p->R || p->rerank > 1024))
        return fail(SCG_ERR_ARG, "rerank shortlist L must be in [R, 1024]");
    if (p->rerank != 0 && h->raw_rows < h->N)
        return fail(SCG_ERR_STATE, "exact distances need the raw vectors (scg_load_raw)");
    switch (p->mode) {
        case SCG_IVFADC:
            if (h->mc != 1 || h->ncells != h->kc) return fail(SCG_ERR_ARG, "This search method is for IVFADC only");
            break;
        case SCG_IMI:
            if (h->mc != 2 || h->ncells != (int64_t)h->kc * h->kc)
                return fail(SCG_ERR_ARG, "This search method is for Multi-D-ADC-2 only");
            break;
        case SCG_SC2:
            if (h->mc != 1 || h->ncells != (int64_t)h->kc * h->kc)
                return fail(SCG_ERR_ARG, "This search method is for MultiRank IVFADC only");
            break;
        case SCG_SC3:
            if (h->mc != 1 || h->kc > 1024 || h->ncells != (int64_t)h->kc * h->kc * h->kc)
                return fail(SCG_ERR_ARG, "This search method is for MultiRank IVFADC-3 only");
            break;
        default:
            return fail(SCG_ERR_ARG, "unknown search mode");
    }
    if (h->kc > 65535) return fail(SCG_ERR_ARG, "kc must be < 65536");
    return SCG_OK;
}

// Per-query tables in the requested arithmetic: the reference's float order
// on CUDA cores, or tcgen05 tensor-core GEMMs (BF16 hi/lo split, one BF16 or
// one FP16 product; FP32 accumulation).
void launch_tables(const TablesArgs &ta, int precision, cudaStream_t s) {
    switch (precision) {
        case SCG_FAST: launch_tables_tc(ta, 3, 1, s); break;
        case SCG_BF16: launch_tables_tc(ta, 1, 1, s); break;
        case SCG_FP16: launch_tables_tc(ta, 1, 0, s); break;
        default: launch_tables_exact(ta, s); break;
    }
}

// The scan's form: exact (the reference's adds) or the fast per-vector form.
int scan_form(int precision) { return precision == SCG_FP32_EXACT ? SCG_FP32_EXACT : SCG_FAST; }

int status_result(int st) {
    if (st & ST_CELL_BUDGET)
        return fail(SCG_ERR_CAP, "a query enumerated more cells than the cell budget; raise it with scg_set_cell_budget");
    if (st & ST_TIE_OVERFLOW) return fail(SCG_ERR_CAP, "too many cells tie exactly at the cut key");
    if (st & ST_ITER_CAP) return fail(SCG_ERR_CAP, "cell selection did not converge within its round cap");
    if (st & ST_TC_TIMEOUT) return fail(SCG_ERR_CUDA, "a tensor-core table tile did not complete in time");
    if (st & ST_BAD_ARG) return fail(SCG_ERR_ARG, "a shortlisted id has no raw vector");
    if (st & ST_POOL) return fail(SCG_ERR_CAP, "the visited-cell pool of the split kernels ran out");
    if (st) return fail(SCG_ERR_CUDA, "search kernel reported status " + std::to_string(st));
    return SCG_OK;
}

int Workspace::init() {
    cudaError_t e = cudaSuccess;
    if (!h_status) e = cudaMallocHost((void **)&h_status, sizeof(int) * 4);
    for (int i = 0; i < 5 && e == cudaSuccess; i++)
        if (!ev[i]) e = cudaEventCreate(&ev[i]);
    if (e != cudaSuccess) return cuda_fail(e, "workspace");
    return SCG_OK;
}

void Workspace::release() {
    DevBuf *all[] = {&dqc, &dqr, &qn, &qsum, &nvis, &empty, &status, &counter, &rec_key, &rec_rank,
                     &rec_cnt, &vis_cell, &vis_pre, &pend, &phase, &sl_ids, &sl_d, &slist, &smeta, &qmeta, &pool_cell, &pool_pre};
    for (DevBuf *b : all) b->release();
    if (h_status) cudaFreeHost(h_status);
    h_status = nullptr;
    for (int i = 0; i < 5; i++)
        if (ev[i]) cudaEventDestroy(ev[i]);
    for (int i = 0; i < 5; i++) ev[i] = nullptr;
}

static size_t up256b(size_t x) { return (x + 255) & ~(size_t)255; }

// Bytes of the sorted coarse lists of nq queries (0 when kc is too large
// for the ahead-of-time sort).
static size_t slist_bytes(int nq, int mc, int kc) {
    return 8ull * nq * (mc == 2 ? 2 : 1) * (size_t)coarse_sort_width(kc);
}

size_t req_bytes(int nq, int dim, int mc, int kc, int mp, int kp, int R, int rerank) {
    (void)dim;
    (void)R;
    size_t b = up256b(4ull * nq * mc * kc) + up256b(4ull * nq * mp * kp) + up256b(8ull * nq) + up256b(4ull * nq) +
               2 * up256b(4ull * nq) + up256b(slist_bytes(nq, mc, kc)) + up256b(8ull * nq * 2);
    if (rerank > 0) b += 2 * up256b(4ull * nq * rerank);
    return b;
}

ReqBufs carve_req(unsigned char *base, int nq, int mc, int kc, int mp, int kp, int rerank) {
    ReqBufs r;
    unsigned char *cur = base;
    auto take = [&](size_t bytes) {
        unsigned char *p = cur;
        cur += up256b(bytes);
        return p;
    };
    r.dqc = (float *)take(4ull * nq * mc * kc);
    r.dqr = (float *)take(4ull * nq * mp * kp);
    r.qn = (float *)take(8ull * nq);
    r.qsum = (float *)take(4ull * nq);
    r.nvis = (int *)take(4ull * nq);
    r.empty = (int *)take(4ull * nq);
    r.sl_ids = nullptr;
    r.sl_d = nullptr;
    r.slist = coarse_sort_width(kc) ? (uint64_t *)take(slist_bytes(nq, mc, kc)) : nullptr;
    r.smeta = (uint32_t *)take(8ull * nq * 2);
    if (rerank > 0) {
        r.sl_ids = (int *)take(4ull * nq * rerank);
        r.sl_d = (float *)take(4ull * nq * rerank);
    }
    return r;
}

int ensure_vterm(scg_index *h, cudaStream_t s) {
    if (h->have_vterm) return SCG_OK;
    int rc;
    // the fast form's per-vector term (one float per database vector)
    if ((rc = h->vterm.ensure(sizeof(float) * (size_t)(h->N ? h->N : 1)))) return rc;
    launch_vterm(index_mode(h), h->kc, h->mp, h->kp, h->mc,
                 (uint64_t)h->ncells, h->N, h->off.as<uint32_t>(), h->codes.as<uint8_t>(), h->norm_r.as<float>(),
                 h->dot_cr.as<float>(), h->vterm.as<float>(), s);
    SCG_CUDA(cudaGetLastError());
    SCG_CUDA(cudaStreamSynchronize(s));
    h->have_vterm = true;
    return SCG_OK;
}

int reserve_search(scg_index *h, Workspace *ws, int mode, int grid) {
    int rc;
    if ((rc = ws->init())) return rc;
    // the largest grid of each slot kind over the kernel variants
    int g_rec = 0, g_vis = 0, g_pend = 0;
    for (int u : {2, 4, 8}) {
        for (int rot : {0, 1}) {
            if (rot && !search_rot_form(SCG_FAST, h->mp, h->kp)) continue;
            const int f = h->num_sms * search_max_blocks_per_sm(mode, h->kc, h->mp, h->kp, u, 0, rot);
            const int c = h->num_sms * search_max_blocks_per_sm(mode, h->kc, h->mp, h->kp, u, 2, rot);
            g_rec = std::max(g_rec, f);
            g_vis = std::max(g_vis, f);
            g_pend = std::max(g_pend, std::max(f, c));
        }
    }
    g_rec = std::max(g_rec, h->num_sms * search_max_blocks_per_sm(mode, h->kc, h->mp, h->kp, 4, 1, 0));
    if (g_rec < 1) return fail(SCG_ERR_ARG, "search kernel does not fit on an SM for this shape");
    if (grid > 0) {
        g_rec = std::min(g_rec, grid);
        g_vis = std::min(g_vis, grid);
        g_pend = std::min(g_pend, grid);
    }
    const size_t slot = (size_t)h->cap_rec, pcap = slot > 65536 ? slot : 65536;
    if ((rc = ws->status.ensure(sizeof(int) * 4))) return rc;
    if ((rc = ws->counter.ensure(sizeof(int) * 4))) return rc;
    if ((rc = ws->rec_key.ensure(4 * slot * g_rec))) return rc;
    if ((rc = ws->rec_rank.ensure(4 * slot * g_rec))) return rc;
    if ((rc = ws->rec_cnt.ensure(4 * slot * g_rec))) return rc;
    if ((rc = ws->vis_cell.ensure(4 * (slot + 1) * g_vis))) return rc;
    if ((rc = ws->vis_pre.ensure(4 * (slot + 1) * g_vis))) return rc;
    if ((rc = ws->pend.ensure(8 * pcap * g_pend))) return rc;
    return SCG_OK;
}

// Pool of the split kernels' visited lists: each query owns POOL_SLOT
// entries (or fewer when T, w or N bound its list below that: each visited
// non-empty cell holds a candidate, so a list has at most min(T, w, N) cells
// plus its closing prefix); longer lists take a range of a shared overflow
// area (64 entries per query, 128 with per-query targets, whose long lists
// the host cannot bound; 65,536 at least).  Should that run out, the batch
// is searched again by the fused kernel, which stalls a request loop, so
// the area is generous (8 bytes per entry).
constexpr int64_t POOL_SLOT = 128;

static void pool_dims(const scg_index *h, const scg_search_params *p, int nq, bool per_query_T, int64_t *stride,
                      int64_t *over) {
    int64_t b = POOL_SLOT - 1;
    if (p) {
        if (!per_query_T) b = std::min<int64_t>(b, p->T > 0 ? (int64_t)p->T : 1);
        b = std::min<int64_t>(b, p->w > 0 ? (int64_t)p->w : 1);
    }
    b = std::min<int64_t>(b, h->N > 0 ? h->N : 1);
    *stride = b + 1;
    *over = std::max<int64_t>(65536, (per_query_T ? 128 : 64) * (int64_t)nq);
}

// Every per-query buffer of the split kernels for batches of up to nq
// queries: the visited-list pool, the deferred-query list and the survivors
// handed to the merge kernel.  The request loop reserves them per slot when
// it starts, so that no request grows a workspace (a cudaFree waits for the
// whole device, every other slot included).
int reserve_pool(scg_index *h, Workspace *ws, int nq) {
    int64_t stride, over;
    pool_dims(h, nullptr, nq, false, &stride, &over);
    int rc;
    if ((rc = ws->qmeta.ensure(sizeof(QMeta) * (size_t)nq))) return rc;
    if ((rc = ws->pool_cell.ensure(4 * (size_t)(stride * nq + over)))) return rc;
    if ((rc = ws->pool_pre.ensure(4 * (size_t)(stride * nq + over)))) return rc;
    if ((rc = ws->defer.ensure(sizeof(int) * ((size_t)nq + 1)))) return rc;
    if ((rc = ws->surv.ensure(sizeof(uint64_t) * (size_t)nq * SURV_CAP))) return rc;
    if ((rc = ws->surv_n.ensure(sizeof(int) * (size_t)nq))) return rc;
    return SCG_OK;
}

int index_mode(const scg_index *h) {
    if (h->mc == 2) return SCG_IMI;
    if (h->ncells == h->kc) return SCG_IVFADC;
    return h->ncells == (int64_t)h->kc * h->kc ? SCG_SC2 : SCG_SC3;
}

int run_search(scg_index *h, Workspace *ws, const ReqBufs *rb, const scg_search_params *p, const float *dQ, int nq,
               int *d_ids, float *d_d, int *d_sums, cudaStream_t s, bool wait, int *h_stat, bool allow_split) {
    int rc;
    if ((rc = ws->init())) return rc;
    // with a shortlist re-rank the ADC search keeps L candidates per query
    const bool rr = p->rerank > 0;
    const int R = rr ? p->rerank : p->R;
    ReqBufs b;
    if (rb) {
        b = *rb;
    } else {
        if ((rc = ws->dqc.ensure(sizeof(float) * (size_t)nq * h->mc * h->kc))) return rc;
        if ((rc = ws->dqr.ensure(sizeof(float) * (size_t)nq * h->mp * h->kp))) return rc;
        if ((rc = ws->qn.ensure(sizeof(float) * (size_t)nq * 2))) return rc;
        if ((rc = ws->qsum.ensure(sizeof(float) * (size_t)nq))) return rc;
        if ((rc = ws->nvis.ensure(sizeof(int) * (size_t)nq))) return rc;
        if ((rc = ws->empty.ensure(sizeof(int) * (size_t)nq))) return rc;
        b.dqc = ws->dqc.as<float>(); b.dqr = ws->dqr.as<float>();
        b.qn = ws->qn.as<float>(); b.qsum = ws->qsum.as<float>();
        b.nvis = ws->nvis.as<int>(); b.empty = ws->empty.as<int>();
        b.sl_ids = nullptr; b.sl_d = nullptr;
        b.slist = nullptr;
        b.smeta = nullptr;
        if (coarse_sort_width(h->kc)) {
            if ((rc = ws->slist.ensure(slist_bytes(nq, h->mc, h->kc)))) return rc;
            if ((rc = ws->smeta.ensure(8ull * nq * 2))) return rc;
            b.slist = ws->slist.as<uint64_t>();
            b.smeta = ws->smeta.as<uint32_t>();
        }
        if (rr) {
            if ((rc = ws->sl_ids.ensure(sizeof(int) * (size_t)nq * R))) return rc;
            if ((rc = ws->sl_d.ensure(sizeof(float) * (size_t)nq * R))) return rc;
            b.sl_ids = ws->sl_ids.as<int>(); b.sl_d = ws->sl_d.as<float>();
        }
    }
    int *s_ids = rr ? b.sl_ids : d_ids;
    float *s_d = rr ? b.sl_d : d_d;
    if ((rc = ws->status.ensure(sizeof(int) * 4))) return rc;
    if ((rc = ws->counter.ensure(sizeof(int) * 4))) return rc;
    const int upl = h->tuned_upl[scan_form(p->precision) == SCG_FAST ? 1 : 0];
    // rerank = -1: the scan scores every candidate by its exact distance
    const int qdim = p->rerank < 0 ? h->dim : 0;
    const int rot = (!qdim && search_rot_form(scan_form(p->precision), h->mp, h->kp)) ? 1 : 0;
    const int *Tq = rb ? nullptr : h->d_Tq;
    // split kernels (selection, then a lighter scan at higher occupancy)
    int64_t stride = 0, over = 0;
    pool_dims(h, p, nq, Tq != nullptr, &stride, &over);
    // the three-list walk of SCG_SC3 runs in the fused kernel only
    const bool split = allow_split && h->split && p->mode != SCG_SC3 && stride * (int64_t)nq + over < (1ll << 32);
    auto grid_of = [&](int part) {
        int g = h->num_sms * search_max_blocks_per_sm(p->mode, h->kc, h->mp, h->kp, upl, part, rot, qdim);
        return std::max(1, std::min(g, nq));
    };
    const int g_fused = split ? 0 : grid_of(0);
    const int g_sel = split ? grid_of(1) : 0, g_scan = split ? grid_of(2) : 0;
    if (std::max(g_fused, std::max(g_sel, g_scan)) < 1)
        return fail(SCG_ERR_ARG, "search kernel does not fit on an SM for this shape");
    size_t slot = (size_t)h->cap_rec;
    const int g_rec = std::max(g_fused, g_sel), g_pend = std::max(g_fused, g_scan);
    if ((rc = ws->rec_key.ensure(4 * slot * g_rec))) return rc;
    if ((rc = ws->rec_rank.ensure(4 * slot * g_rec))) return rc;
    if ((rc = ws->rec_cnt.ensure(4 * slot * g_rec))) return rc;
    if (!split) {
        if ((rc = ws->vis_cell.ensure(4 * (slot + 1) * g_fused))) return rc;
        if ((rc = ws->vis_pre.ensure(4 * (slot + 1) * g_fused))) return rc;
    } else {
        if ((rc = ws->qmeta.ensure(sizeof(QMeta) * (size_t)nq))) return rc;
        if ((rc = ws->pool_cell.ensure(4 * (size_t)(stride * nq + over)))) return rc;
        if ((rc = ws->pool_pre.ensure(4 * (size_t)(stride * nq + over)))) return rc;
    }
    // the selection of the split search: one warp per query where it serves
    // the shape, the block-wide kernel for the rest (and every other shape)
    const bool warp_sel = split && b.slist && select_warp_serves(p->mode, h->kc);
    if (warp_sel && (rc = ws->defer.ensure(sizeof(int) * ((size_t)nq + 1)))) return rc;
    // the top-R of the split scan: one warp per query in a merge kernel
    // (outputs in order, R <= 256), else inside the scan kernel
    const bool warp_merge = split && !rr && R <= 256;
    if (warp_merge && ((rc = ws->surv.ensure(sizeof(uint64_t) * (size_t)nq * SURV_CAP)) ||
                       (rc = ws->surv_n.ensure(sizeof(int) * (size_t)nq))))
        return rc;
    // survivors of the scan's threshold, per resident CTA
    const size_t pcap = slot > 65536 ? slot : 65536;
    if ((rc = ws->pend.ensure(8 * pcap * g_pend))) return rc;

    // kernels this call launches (scg_last_launches)
    int nl = 0;
    if (scan_form(p->precision) == SCG_FAST) {
        const bool had_vterm = h->have_vterm;
        if ((rc = ensure_vterm(h, s))) return rc;
        if (!had_vterm) nl++;
    }
    TablesArgs ta;
    memset(&ta, 0, sizeof(ta));
    ta.dim = h->dim; ta.mc = h->mc; ta.kc = h->kc; ta.mp = h->mp; ta.kp = h->kp; ta.nq = nq;
    ta.Q = dQ;
    ta.cq = h->cq.as<float>(); ta.pq = h->pq.as<float>();
    ta.norm_c = h->norm_c.as<float>(); ta.norm_r = h->norm_r.as<float>();
    ta.dqc = b.dqc; ta.dqr = b.dqr;
    ta.qn = b.qn; ta.qsum = b.qsum;
    ta.lut_only = scan_form(p->precision) == SCG_FAST;
    ta.status = ws->status.as<int>();
    SCG_CUDA(cudaMemsetAsync(ws->status.p, 0, sizeof(int) * 4, s));
    SCG_CUDA(cudaMemsetAsync(ws->counter.p, 0, sizeof(int) * 4, s));
    SCG_CUDA(cudaEventRecord(ws->ev[0], s));
    launch_tables(ta, p->precision, s);
    if (nq > 0) nl += 2;  // the tables and the query norms
    if (b.slist) {
        CoarseArgs ca;
        ca.dqc = b.dqc; ca.qn = b.qn; ca.qsum = b.qsum;
        ca.nq = nq; ca.kc = h->kc; ca.mc = h->mc; ca.imi = h->mc == 2 ? 1 : 0;
        ca.Tq = rb ? nullptr : h->d_Tq;
        ca.T = p->T;
        ca.avg_density = (double)h->N / (double)(h->ncells ? h->ncells : 1);
        ca.dens_acc = h->dens.as<unsigned long long>();
        ca.max_prefix = 1024;
        ca.fixed_prefix = h->prefix_len;
        ca.width = coarse_sort_width(h->kc);
        ca.out = b.slist;
        ca.meta = b.smeta;
        launch_coarse_prefix(ca, s);
        if (nq > 0) nl++;
    }
    SCG_CUDA(cudaEventRecord(ws->ev[1], s));

    SearchArgs sa;
    memset(&sa, 0, sizeof(sa));
    sa.mode = p->mode; sa.dim = h->dim; sa.mc = h->mc; sa.kc = h->kc; sa.mp = h->mp; sa.kp = h->kp;
    sa.nq = nq; sa.R = R; sa.w = p->w; sa.T = p->T; sa.precision = scan_form(p->precision);
    sa.rot = rot;
    sa.raw_dim = qdim;
    sa.Q = dQ;
    sa.raw = qdim ? h->raw.p : nullptr;
    sa.raw_u8 = h->raw_u8 ? 1 : 0;
    sa.upl = upl;
    sa.slist = b.slist;
    sa.smeta = b.smeta;
    sa.slist_w = coarse_sort_width(h->kc);
    sa.Tq = Tq;
    sa.rank_limit = h->rank_limit;
    sa.dqc = b.dqc; sa.dqr = b.dqr; sa.qn = b.qn; sa.qsum = b.qsum;
    sa.off = h->off.as<uint32_t>(); sa.pid = h->pid.as<int>(); sa.codes = h->codes.as<uint8_t>();
    sa.dot_cr = h->dot_cr.as<float>();
    sa.vterm = h->vterm.as<float>();
    sa.ncells = (uint64_t)h->ncells;
    sa.N = h->N;
    sa.rec_key = ws->rec_key.as<uint32_t>(); sa.rec_rank = ws->rec_rank.as<uint32_t>();
    sa.rec_cnt = ws->rec_cnt.as<uint32_t>();
    sa.vis_cell = split ? nullptr : ws->vis_cell.as<uint32_t>();
    sa.vis_pre = split ? nullptr : ws->vis_pre.as<uint32_t>();
    sa.qmeta = split ? ws->qmeta.as<QMeta>() : nullptr;
    sa.pool_cell = split ? ws->pool_cell.as<uint32_t>() : nullptr;
    sa.pool_pre = split ? ws->pool_pre.as<uint32_t>() : nullptr;
    sa.pool_stride = split ? (uint32_t)stride : 0u;
    sa.pool_over = ws->counter.as<uint32_t>() + 2;
    sa.pool_over_cap = split ? (uint32_t)over : 0u;
    sa.cap_rec = h->cap_rec;
    sa.pend = ws->pend.as<uint64_t>();
    sa.pcap = (uint32_t)pcap;
    sa.qcounter = ws->counter.as<int>();
    sa.out_ids = s_ids; sa.out_d = s_d; sa.out_sum = d_sums;
    sa.shortlist = rr ? 1 : 0;
    sa.out_nvis = b.nvis; sa.out_empty = b.empty;
    sa.status = ws->status.as<int>();
    sa.phase_cycles = nullptr;
    sa.dens_acc = h->dens.as<unsigned long long>();
    if (ws->phase_on) {
        if ((rc = ws->phase.ensure(sizeof(long long) * 16))) return rc;
        SCG_CUDA(cudaMemsetAsync(ws->phase.p, 0, sizeof(long long) * 16, s));
        sa.phase_cycles = ws->phase.as<long long>();
    }
    if (nq > 0) {
        if (split) {
            // persistent launches, each with its own query counter
            if (warp_sel) {
                SCG_CUDA(cudaMemsetAsync(ws->defer.p, 0, sizeof(int), s));
                sa.qcounter = ws->counter.as<int>() + 3;
                const int gw = h->num_sms * std::max(1, select_warp_blocks_per_sm());
                if (select_warp_launch(sa, ws->defer.as<int>(), std::max(1, std::min(gw, (nq + 3) / 4)), s))
                    return fail(SCG_ERR_CUDA, "warp-wide selection launch failed");
                sa.qlist = ws->defer.as<int>();
                nl++;
            }
            sa.qcounter = ws->counter.as<int>();
            if ((rc = search_launch(sa, 1, g_sel, s))) return rc;
            nl++;
            sa.qlist = nullptr;
            SCG_CUDA(cudaEventRecord(ws->ev[4], s));
            sa.qcounter = ws->counter.as<int>() + 1;
            if (warp_merge) {
                sa.surv = ws->surv.as<uint64_t>();
                sa.surv_n = ws->surv_n.as<int>();
                sa.surv_cap = SURV_CAP;
            }
            if ((rc = search_launch(sa, 2, g_scan, s))) return rc;
            nl++;
            if (warp_merge) {
                merge_warp_launch(sa.surv, sa.surv_n, SURV_CAP, sa.pid, nq, R, s_ids, s_d, h->num_sms, s);
                SCG_CUDA(cudaGetLastError());
                nl++;
            }
        } else if ((rc = search_launch(sa, 0, g_fused, s))) {
            return rc;
        } else {
            nl++;
        }
    }
    SCG_CUDA(cudaEventRecord(ws->ev[2], s));
    if (rr && nq > 0) {
        if (rerank_smem_bytes(R, h->dim) > 227 * 1024) return fail(SCG_ERR_ARG, "dimension too large for the re-rank");
        launch_rerank(dQ, nq, h->dim, h->raw.p, h->raw_u8 ? 1 : 0, h->raw_rows, s_ids, R, p->R, d_ids, d_d,
                      ws->status.as<int>(), s);
        SCG_CUDA(cudaGetLastError());
        nl++;
    }
    SCG_CUDA(cudaEventRecord(ws->ev[3], s));
    ws->last_nq = nq;
    ws->last_split = split && nq > 0;
    ws->last_launches = nl;
    int *dst = h_stat ? h_stat : ws->h_status;
    SCG_CUDA(cudaMemcpyAsync(dst, ws->status.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    if (!wait) return SCG_OK;
    SCG_CUDA(cudaStreamSynchronize(s));
    if (split && (*dst & ST_POOL)) {  // the visited lists outgrew the pool
        rc = run_search(h, ws, rb, p, dQ, nq, d_ids, d_d, d_sums, s, true, h_stat, false);
        ws->last_launches += nl;
        return rc;
    }
    return status_result(*dst);
}

}  // namespace scg

extern "C" {

int scg_last_error(char *buf, int len) {
    if (!buf || len <= 0) return SCG_ERR_ARG;
    snprintf(buf, (size_t)len, "%s", g_err.c_str());
    return SCG_OK;
}

int scg_index_create(scg_index **out, int device) {
    if (!out) return fail(SCG_ERR_ARG, "null output pointer");
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDeviceCount");
    if (device < 0 || device >= n) return fail(SCG_ERR_ARG, "no such CUDA device");
    scg_index *h = new scg_index();
    h->device = device;
    e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete h;
        return cuda_fail(e, "scg_index_create");
    }
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->stream2, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMallocHost((void **)&h->h_chunk_status, sizeof(int) * 8);
    int rc = e == cudaSuccess ? h->ws.init() : cuda_fail(e, "scg_index_create");
    if (rc == SCG_OK) rc = h->ws2.init();
    if (rc) {
        h->ws.release();
        h->ws2.release();
        if (h->h_chunk_status) cudaFreeHost(h->h_chunk_status);
        if (h->stream2) cudaStreamDestroy(h->stream2);
        cudaStreamDestroy(h->stream);
        delete h;
        return rc;
    }
    *out = h;
    return SCG_OK;
}

int scg_index_destroy(scg_index *h) {
    if (!h) return SCG_OK;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    DevBuf *all[] = {&h->cq, &h->pq, &h->norm_c, &h->norm_r, &h->dot_cr, &h->off, &h->pid, &h->codes,
                     &h->raw, &h->vterm, &h->q, &h->ids, &h->dists, &h->sums, &h->reqbuf,
                     &h->enc_nc, &h->enc_nr, &h->enc_cmax, &h->enc_rmax, &h->enc_tab, &h->enc_res,
                     &h->enc_status};
    for (DevBuf *b : all) b->release();
    if (h->stream2) cudaStreamSynchronize(h->stream2);
    if (h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
    h->ws.release();
    h->ws2.release();
    if (h->h_chunk_status) cudaFreeHost(h->h_chunk_status);
    if (h->stream2) cudaStreamDestroy(h->stream2);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return SCG_OK;
}

int scg_load_codebooks(scg_index *h, const float *cq, int kc, int mc, const float *pq, int kp, int mp, int dim) {
    if (!h || !cq || !pq) return fail(SCG_ERR_ARG, "null argument");
    if (kc <= 0 || mc <= 0 || kp <= 0 || mp <= 0 || dim <= 0) return fail(SCG_ERR_ARG, "non-positive shape");
    if (dim % mc || dim % mp || mp % mc) return fail(SCG_ERR_ARG, "dim must divide by mc and mp, mp by mc");
    if (mc > 2) return fail(SCG_ERR_ARG, "mc must be 1 or 2");
    if (kp > 256) return fail(SCG_ERR_ARG, "kp must be <= 256 (uint8 codes)");
    std::lock_guard<std::mutex> g(h->mu);
    int rc;
    if ((rc = set_device(h))) return rc;
    if ((rc = h->cq.ensure(sizeof(float) * (size_t)kc * dim))) return rc;
    if ((rc = h->pq.ensure(sizeof(float) * (size_t)kp * dim))) return rc;
    SCG_CUDA(copy_in(h->cq.p, cq, sizeof(float) * (size_t)kc * dim, h->stream));
    SCG_CUDA(copy_in(h->pq.p, pq, sizeof(float) * (size_t)kp * dim, h->stream));
    h->dim = dim; h->mc = mc; h->kc = kc; h->mp = mp; h->kp = kp;
    h->have_codebooks = true;
    h->enc_ready = false;
    h->precomputed = false;
    h->have_vterm = false;
    return SCG_OK;
}

int scg_load_codebooks_file(scg_index *h, const char *cq_path, const char *pq_path) {
    std::vector<float> c, p;
    int kc, mc, dc, kp, mp, dp, rc;
    if ((rc = read_ctr(cq_path, c, kc, mc, dc))) return rc;
    if ((rc = read_ctr(pq_path, p, kp, mp, dp))) return rc;
    if (dc != dp) return fail(SCG_ERR_IO, "codebook dimensions differ");
    return scg_load_codebooks(h, c.data(), kc, mc, p.data(), kp, mp, dc);
}

int scg_load_csr(scg_index *h, const int *L, const int *pid, const uint8_t *codes, int64_t N, int64_t ncells) {
    if (!h || !L || (N > 0 && (!pid || !codes))) return fail(SCG_ERR_ARG, "null argument");
    if (!h->have_codebooks) return fail(SCG_ERR_STATE, "load codebooks before encoded data");
    if (N < 0 || N > 0xfffffffeLL) return fail(SCG_ERR_ARG, "N out of range");
    int64_t imi_cells = ipow(h->kc, h->mc), sc_cells = (int64_t)h->kc * h->kc, sc3_cells = sc_cells * h->kc;
    if (ncells != imi_cells && !(h->mc == 1 && (ncells == sc_cells || (ncells == sc3_cells && h->kc <= 1024))))
        return fail(SCG_ERR_ARG, "ncells must be kc^mc, kc^2 or kc^3 (second candidate, kc <= 1024)");
    std::vector<uint32_t> off((size_t)ncells + 1);
    off[0] = 0;
    int prev = 0;
    for (int64_t c = 0; c < ncells; c++) {
        if (L[c] < prev) return fail(SCG_ERR_ARG, "L must be a non-decreasing inclusive prefix");
        prev = L[c];
        off[(size_t)c + 1] = (uint32_t)L[c];
    }
    if ((int64_t)prev != N) return fail(SCG_ERR_ARG, "L[ncells-1] must equal N");
    for (int64_t i = 0; i < N * h->mp; i++)
        if (codes[i] >= h->kp) return fail(SCG_ERR_ARG, "a code is not below kp");
    for (int64_t i = 0; i < N; i++)
        if (pid[i] < 0) return fail(SCG_ERR_ARG, "negative pid");
    std::lock_guard<std::mutex> g(h->mu);
    int rc;
    if ((rc = set_device(h))) return rc;
    if ((rc = h->off.ensure(sizeof(uint32_t) * off.size()))) return rc;
    if ((rc = h->pid.ensure(sizeof(int) * (size_t)(N ? N : 1)))) return rc;
    if ((rc = h->codes.ensure((size_t)(N ? N : 1) * h->mp))) return rc;
    SCG_CUDA(copy_in(h->off.p, off.data(), sizeof(uint32_t) * off.size(), h->stream));
    if (N) {
        SCG_CUDA(copy_in(h->pid.p, pid, sizeof(int) * (size_t)N, h->stream));
        SCG_CUDA(copy_in(h->codes.p, codes, (size_t)N * h->mp, h->stream));
    }
    h->N = N;
    h->ncells = ncells;
    h->have_csr = true;
    if (h->dens.p) SCG_CUDA(cudaMemset(h->dens.p, 0, 16));
    h->have_vterm = false;
    return SCG_OK;
}

int scg_load_encoded_file(scg_index *h, const char *path, int nc) {
    if (!h || !path) return fail(SCG_ERR_ARG, "null argument");
    if (!h->have_codebooks) return fail(SCG_ERR_STATE, "load codebooks before encoded data");
    int64_t ncells = ipow(h->kc, nc);
    std::vector<unsigned char> b;
    if (!read_file(path, b)) return fail(SCG_ERR_IO, std::string("cannot read ") + path);
    if (b.size() < 8) return fail(SCG_ERR_IO, "encoded file too short");
    int hdr[2];
    memcpy(hdr, b.data(), 8);
    int64_t N = hdr[1];
    if (N < 0) return fail(SCG_ERR_IO, "negative N in encoded file");
    std::vector<int> L((size_t)ncells), pid((size_t)(N ? N : 1));
    std::vector<uint8_t> codes((size_t)(N ? N : 1) * h->mp);
    size_t pos = 8;
    int64_t base = 0, acc = 0;
    for (int64_t c = 0; c < ncells; c++) {
        if (pos + 4 > b.size()) return fail(SCG_ERR_IO, "encoded file truncated (cell lengths)");
        int l;
        memcpy(&l, b.data() + pos, 4);
        pos += 4;
        if (l < 0 || base + l > N) return fail(SCG_ERR_IO, "encoded file: bad cell length");
        if (l > 0) {
            size_t need = (size_t)l * 4 + (size_t)l * h->mp;
            if (pos + need > b.size()) return fail(SCG_ERR_IO, "encoded file truncated (cell data)");
            memcpy(pid.data() + base, b.data() + pos, (size_t)l * 4);
            pos += (size_t)l * 4;
            memcpy(codes.data() + base * h->mp, b.data() + pos, (size_t)l * h->mp);
            pos += (size_t)l * h->mp;
            base += l;
        }
        acc += l;
        L[(size_t)c] = (int)acc;
    }
    if (base != N) return fail(SCG_ERR_IO, "encoded file: cell lengths do not sum to N");
    return scg_load_csr(h, L.data(), pid.data(), codes.data(), N, ncells);
}

static int load_raw(scg_index *h, const void *X, int64_t N, size_t elem, bool u8) {
    if (!h || (N > 0 && !X)) return fail(SCG_ERR_ARG, "null argument");
    if (N < 0) return fail(SCG_ERR_ARG, "N < 0");
    if (!h->have_codebooks) return fail(SCG_ERR_STATE, "load codebooks first");
    std::lock_guard<std::mutex> g(h->mu);
    int rc;
    if ((rc = set_device(h))) return rc;
    const size_t bytes = elem * (size_t)N * h->dim;
    if ((rc = h->raw.ensure(bytes ? bytes : 16))) return rc;
    if (bytes) SCG_CUDA(copy_in(h->raw.p, X, bytes, h->stream));
    h->raw_rows = N;
    h->raw_u8 = u8;
    return SCG_OK;
}

int scg_load_raw(scg_index *h, const float *X, int64_t N) { return load_raw(h, X, N, sizeof(float), false); }

int scg_load_raw_u8(scg_index *h, const uint8_t *X, int64_t N) { return load_raw(h, X, N, 1, true); }

int scg_precompute(scg_index *h) {
    if (!h) return fail(SCG_ERR_ARG, "null index");
    if (!h->have_codebooks) return fail(SCG_ERR_STATE, "codebooks not loaded");
    std::lock_guard<std::mutex> g(h->mu);
    int rc;
    if ((rc = set_device(h))) return rc;
    if ((rc = h->norm_c.ensure(sizeof(float) * (size_t)h->mc * h->kc))) return rc;
    if ((rc = h->norm_r.ensure(sizeof(float) * (size_t)h->mp * h->kp))) return rc;
    if ((rc = h->dot_cr.ensure(sizeof(float) * (size_t)h->kc * h->kp * h->mp))) return rc;
    launch_precompute1(h->dim, h->mc, h->kc, h->mp, h->kp, h->cq.as<float>(), h->pq.as<float>(),
                       h->norm_c.as<float>(), h->norm_r.as<float>(), h->dot_cr.as<float>(), h->stream);
    SCG_CUDA(cudaGetLastError());
    SCG_CUDA(cudaStreamSynchronize(h->stream));
    if ((rc = h->dens.ensure(16))) return rc;
    SCG_CUDA(cudaMemset(h->dens.p, 0, 16));
    h->precomputed = true;
    h->have_vterm = false;
    return SCG_OK;
}

int scg_search_device(scg_index *h, const scg_search_params *p, const float *dQ, int nq, int *d_ids, float *d_dists,
                      int *d_sums, void *stream) {
    int rc;
    if ((rc = check_ready(h))) return rc;
    if ((rc = check_params(h, p, nq))) return rc;
    if (nq > 0 && (!dQ || !d_ids || !d_dists || !d_sums)) return fail(SCG_ERR_ARG, "null buffer");
    std::lock_guard<std::mutex> g(h->mu);
    if ((rc = set_device(h))) return rc;
    cudaStream_t s = stream ? (cudaStream_t)stream : h->stream;
    return run_search(h, &h->ws, nullptr, p, dQ, nq, d_ids, d_dists, d_sums, s, true);
}

// Smallest chunk of the host-buffer search with page-locked and with
// pageable buffers (at most 4 chunks per batch).
#ifndef SCG_HOST_CHUNK_PINNED
#define SCG_HOST_CHUNK_PINNED 2048
#endif
#ifndef SCG_HOST_CHUNK_MIN
#define SCG_HOST_CHUNK_MIN 1024
#endif

int scg_search(scg_index *h, const scg_search_params *p, const float *Q, int nq, int *ids, float *dists, int *sums) {
    int rc;
    if ((rc = check_ready(h))) return rc;
    if ((rc = check_params(h, p, nq))) return rc;
    if (nq > 0 && (!Q || !ids || !dists)) return fail(SCG_ERR_ARG, "null buffer");
    std::lock_guard<std::mutex> g(h->mu);
    if ((rc = set_device(h))) return rc;
    if (nq == 0) return SCG_OK;
    const int R = p->R;
    if ((rc = h->q.ensure(sizeof(float) * (size_t)nq * h->dim))) return rc;
    if ((rc = h->ids.ensure(sizeof(int) * (size_t)nq * R))) return rc;
    if ((rc = h->dists.ensure(sizeof(float) * (size_t)nq * R))) return rc;
    if ((rc = h->sums.ensure(sizeof(int) * (size_t)nq))) return rc;
    if ((rc = h->ws.nvis.ensure(sizeof(int) * (size_t)nq))) return rc;
    if ((rc = h->ws.empty.ensure(sizeof(int) * (size_t)nq))) return rc;
    // The batch runs in chunks alternating over two streams (each with its
    // own workspace), so that one chunk's copies overlap another chunk's
    // search and the next chunk's kernels fill the tail of the previous
    // one's.  With page-locked caller buffers every chunk copies its results
    // out as soon as it is done; with pageable buffers (staged copies that
    // block the host) every chunk is enqueued before the first copy-out.
    auto pinned = [](const void *ptr) {
        if (!ptr) return true;
        cudaPointerAttributes at;
        if (cudaPointerGetAttributes(&at, ptr) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        return at.type == cudaMemoryTypeHost;
    };
    const bool eager_out = pinned(ids) && pinned(dists) && pinned(sums);
    const bool q_pinned = pinned(Q);
    const int nch = std::max(1, std::min(4, nq / ((eager_out && q_pinned) ? SCG_HOST_CHUNK_PINNED : SCG_HOST_CHUNK_MIN)));
    const int per = (nq + nch - 1) / nch;
    size_t off_b[8];
    size_t total = 0;
    for (int c = 0; c < nch; c++) {
        const int n = std::min(per, nq - c * per);
        off_b[c] = total;
        total += req_bytes(n, h->dim, h->mc, h->kc, h->mp, h->kp, R, p->rerank);
    }
    if ((rc = h->reqbuf.ensure(total))) return rc;
    cudaStream_t ss[2] = {h->stream, h->stream2};
    Workspace *ww[2] = {&h->ws, &h->ws2};
    for (int c = 0; c < nch; c++) {
        const int q0 = c * per, n = std::min(per, nq - q0);
        cudaStream_t s = ss[c & 1];
        ReqBufs rb = carve_req(h->reqbuf.as<unsigned char>() + off_b[c], n, h->mc, h->kc, h->mp, h->kp, p->rerank);
        float *dq = h->q.as<float>() + (size_t)q0 * h->dim;
        SCG_CUDA(cudaMemcpyAsync(dq, Q + (size_t)q0 * h->dim, sizeof(float) * (size_t)n * h->dim,
                                 cudaMemcpyHostToDevice, s));
        h->h_chunk_status[c] = 0;
        rc = run_search(h, ww[c & 1], &rb, p, dq, n, h->ids.as<int>() + (size_t)q0 * R,
                        h->dists.as<float>() + (size_t)q0 * R, h->sums.as<int>() + q0, s, false,
                        &h->h_chunk_status[c]);
        if (rc) {
            cudaStreamSynchronize(h->stream);
            cudaStreamSynchronize(h->stream2);
            return rc;
        }
        // per-query facts for scg_last_query_stats, in batch order
        SCG_CUDA(cudaMemcpyAsync(h->ws.nvis.as<int>() + q0, rb.nvis, sizeof(int) * (size_t)n,
                                 cudaMemcpyDeviceToDevice, s));
        SCG_CUDA(cudaMemcpyAsync(h->ws.empty.as<int>() + q0, rb.empty, sizeof(int) * (size_t)n,
                                 cudaMemcpyDeviceToDevice, s));
        if (eager_out) {
            SCG_CUDA(cudaMemcpyAsync(ids + (size_t)q0 * R, h->ids.as<int>() + (size_t)q0 * R,
                                     sizeof(int) * (size_t)n * R, cudaMemcpyDeviceToHost, s));
            SCG_CUDA(cudaMemcpyAsync(dists + (size_t)q0 * R, h->dists.as<float>() + (size_t)q0 * R,
                                     sizeof(float) * (size_t)n * R, cudaMemcpyDeviceToHost, s));
            if (sums)
                SCG_CUDA(cudaMemcpyAsync(sums + q0, h->sums.as<int>() + q0, sizeof(int) * (size_t)n,
                                         cudaMemcpyDeviceToHost, s));
        }
    }
    for (int c = 0; c < nch && !eager_out; c++) {
        const int q0 = c * per, n = std::min(per, nq - q0);
        cudaStream_t s = ss[c & 1];
        SCG_CUDA(cudaMemcpyAsync(ids + (size_t)q0 * R, h->ids.as<int>() + (size_t)q0 * R, sizeof(int) * (size_t)n * R,
                                 cudaMemcpyDeviceToHost, s));
        SCG_CUDA(cudaMemcpyAsync(dists + (size_t)q0 * R, h->dists.as<float>() + (size_t)q0 * R,
                                 sizeof(float) * (size_t)n * R, cudaMemcpyDeviceToHost, s));
        if (sums)
            SCG_CUDA(cudaMemcpyAsync(sums + q0, h->sums.as<int>() + q0, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, s));
    }
    SCG_CUDA(cudaStreamSynchronize(h->stream));
    SCG_CUDA(cudaStreamSynchronize(h->stream2));
    h->ws.last_nq = nq;
    for (int c = 0; c < nch; c++) {
        if (h->h_chunk_status[c] == ST_POOL) {
            // this chunk's visited lists outgrew the pool: search it again fused
            const int q0 = c * per, n = std::min(per, nq - q0);
            cudaStream_t s = h->stream;
            ReqBufs rb = carve_req(h->reqbuf.as<unsigned char>() + off_b[c], n, h->mc, h->kc, h->mp, h->kp, p->rerank);
            rc = run_search(h, &h->ws, &rb, p, h->q.as<float>() + (size_t)q0 * h->dim, n,
                            h->ids.as<int>() + (size_t)q0 * R, h->dists.as<float>() + (size_t)q0 * R,
                            h->sums.as<int>() + q0, s, true, &h->h_chunk_status[c], false);
            if (rc) return rc;
            SCG_CUDA(cudaMemcpy(ids + (size_t)q0 * R, h->ids.as<int>() + (size_t)q0 * R, sizeof(int) * (size_t)n * R,
                                cudaMemcpyDeviceToHost));
            SCG_CUDA(cudaMemcpy(dists + (size_t)q0 * R, h->dists.as<float>() + (size_t)q0 * R,
                                sizeof(float) * (size_t)n * R, cudaMemcpyDeviceToHost));
            if (sums) SCG_CUDA(cudaMemcpy(sums + q0, h->sums.as<int>() + q0, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost));
            SCG_CUDA(cudaMemcpy(h->ws.nvis.as<int>() + q0, rb.nvis, sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice));
            SCG_CUDA(cudaMemcpy(h->ws.empty.as<int>() + q0, rb.empty, sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice));
        } else if (h->h_chunk_status[c]) {
            return status_result(h->h_chunk_status[c]);
        }
    }
    return SCG_OK;
}

int scg_search_graph(scg_index *h, const scg_search_params *p, const float *dQ, int nq, int *d_ids, float *d_dists,
                     int *d_sums, void *stream) {
    int rc;
    if ((rc = check_ready(h))) return rc;
    if ((rc = check_params(h, p, nq))) return rc;
    if (nq < 1 || !dQ || !d_ids || !d_dists || !d_sums) return fail(SCG_ERR_ARG, "null buffer or empty batch");
    if (!stream) return fail(SCG_ERR_ARG, "scg_search_graph needs a stream of the caller's");
    std::lock_guard<std::mutex> g(h->mu);
    if ((rc = set_device(h))) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    // everything the captured sequence reads or writes, as one key
    char key[512];
    snprintf(key, sizeof(key), "%d %d %d %d %d %d|%p %d %p %p %p|%p %d %d %d %d %lld %d %d", p->mode, p->R, p->w,
             p->T, p->precision, p->rerank, (const void *)dQ, nq, (void *)d_ids, (void *)d_dists, (void *)d_sums,
             (const void *)h->d_Tq, (int)h->split, h->tuned_upl[0], h->tuned_upl[1], h->cap_rec, (long long)h->N,
             h->device, h->rank_limit * 4096 + h->prefix_len);
    if (!h->graph_exec || h->graph_key != key || h->graph_stream != s) {
        if (h->graph_exec) {
            cudaGraphExecDestroy(h->graph_exec);
            h->graph_exec = nullptr;
        }
        // one ordinary run sizes every buffer and builds the per-vector term,
        // so that nothing allocates or synchronises inside the capture
        if ((rc = run_search(h, &h->ws, nullptr, p, dQ, nq, d_ids, d_dists, d_sums, s, true))) return rc;
        cudaGraph_t graph = nullptr;
        SCG_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
        rc = run_search(h, &h->ws, nullptr, p, dQ, nq, d_ids, d_dists, d_sums, s, false, nullptr, true);
        cudaError_t e = cudaStreamEndCapture(s, &graph);
        if (rc) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
        e = cudaGraphInstantiate(&h->graph_exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            h->graph_exec = nullptr;
            return cuda_fail(e, "cudaGraphInstantiate");
        }
        h->graph_key = key;
        h->graph_stream = s;
    }
    SCG_CUDA(cudaGraphLaunch(h->graph_exec, s));
    SCG_CUDA(cudaStreamSynchronize(s));
    h->ws.last_nq = nq;
    int st = *h->ws.h_status;
    if (st & ST_POOL)  // the visited lists outgrew the pool: search again fused
        return run_search(h, &h->ws, nullptr, p, dQ, nq, d_ids, d_dists, d_sums, s, true, nullptr, false);
    return status_result(st);
}

int scg_query_tables_device(scg_index *h, int precision, const float *dQ, int nq, float *d_diff_qc, float *d_diff_qr,
                            void *stream) {
    if (!h) return fail(SCG_ERR_ARG, "null index");
    if (!h->have_codebooks) return fail(SCG_ERR_STATE, "codebooks not loaded");
    if (!h->precomputed) return fail(SCG_ERR_STATE, "scg_precompute not called");
    if (precision < SCG_FP32_EXACT || precision > SCG_FP16) return fail(SCG_ERR_ARG, "unknown precision");
    if (nq < 0) return fail(SCG_ERR_ARG, "nq < 0");
    if (nq > 0 && (!dQ || !d_diff_qc || !d_diff_qr)) return fail(SCG_ERR_ARG, "null buffer");
    std::lock_guard<std::mutex> g(h->mu);
    int rc;
    if ((rc = set_device(h))) return rc;
    if (nq == 0) return SCG_OK;
    cudaStream_t s = stream ? (cudaStream_t)stream : h->stream;
    if ((rc = h->ws.status.ensure(sizeof(int) * 4))) return rc;
    SCG_CUDA(cudaMemsetAsync(h->ws.status.p, 0, sizeof(int) * 4, s));
    TablesArgs ta;
    memset(&ta, 0, sizeof(ta));
    ta.dim = h->dim; ta.mc = h->mc; ta.kc = h->kc; ta.mp = h->mp; ta.kp = h->kp; ta.nq = nq;
    ta.Q = dQ;
    ta.cq = h->cq.as<float>(); ta.pq = h->pq.as<float>();
    ta.norm_c = h->norm_c.as<float>(); ta.norm_r = h->norm_r.as<float>();
    ta.dqc = d_diff_qc; ta.dqr = d_diff_qr;
    ta.qn = nullptr; ta.qsum = nullptr;
    ta.lut_only = 0;
    ta.status = h->ws.status.as<int>();
    launch_tables(ta, precision, s);
    SCG_CUDA(cudaGetLastError());
    SCG_CUDA(cudaMemcpyAsync(h->ws.h_status, h->ws.status.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    SCG_CUDA(cudaStreamSynchronize(s));
    if (*h->ws.h_status) return status_result(*h->ws.h_status);
    return SCG_OK;
}

int scg_set_scan_tuning(scg_index *h, int precision, int upl) {
    if (!h) return fail(SCG_ERR_ARG, "null index");
    if (precision < SCG_FP32_EXACT || precision > SCG_FP16) return fail(SCG_ERR_ARG, "unknown precision");
    if (upl != 2 && upl != 4 && upl != 8) return fail(SCG_ERR_ARG, "candidates per lane must be 2, 4 or 8");
    std::lock_guard<std::mutex> g(h->mu);
    h->tuned_upl[scan_form(precision) == SCG_FAST ? 1 : 0] = upl;
    return SCG_OK;
}

int scg_autotune(scg_index *h, const scg_search_params *p, const float *dQ, int nq, int *d_ids, float *d_dists,
                 int *d_sums, int *choice, float *ms) {
    int rc;
    if ((rc = check_ready(h))) return rc;
    if ((rc = check_params(h, p, nq))) return rc;
    if (nq < 1 || !dQ || !d_ids || !d_dists || !d_sums) return fail(SCG_ERR_ARG, "autotune needs a non-empty batch");
    std::lock_guard<std::mutex> g(h->mu);
    if ((rc = set_device(h))) return rc;
    cudaStream_t s = h->stream;
    const int form = scan_form(p->precision) == SCG_FAST ? 1 : 0;
    const int saved = h->tuned_upl[form];
    const int cand[3] = {2, 4, 8};
    float best = 3.4e38f;
    int pick = saved;
    for (int i = 0; i < 3; i++) {
        h->tuned_upl[form] = cand[i];
        float t = 3.4e38f;
        for (int rep = 0; rep < 3; rep++) {  // first run warms up
            if ((rc = run_search(h, &h->ws, nullptr, p, dQ, nq, d_ids, d_dists, d_sums, s, true))) {
                h->tuned_upl[form] = saved;
                return rc;
            }
            float k = 0;
            SCG_CUDA(cudaEventElapsedTime(&k, h->ws.ev[1], h->ws.ev[2]));
            if (rep > 0 && k < t) t = k;
        }
        if (ms) ms[i] = t;
        if (t < best) {
            best = t;
            pick = cand[i];
        }
    }
    h->tuned_upl[form] = pick;
    if (choice) *choice = pick;
    return SCG_OK;
}

// Best device time (ms) of the selection + scan of `reps` - 1 searches after
// one warm-up search.
static int tune_time(scg_index *h, const scg_search_params *p, const float *dQ, int nq, int *d_ids, float *d_dists,
                     int *d_sums, int reps, float *ms) {
    float t = 3.4e38f;
    for (int rep = 0; rep < reps; rep++) {
        int rc = run_search(h, &h->ws, nullptr, p, dQ, nq, d_ids, d_dists, d_sums, h->stream, true);
        if (rc) return rc;
        float a = 0, b = 0;
        SCG_CUDA(cudaEventElapsedTime(&a, h->ws.ev[0], h->ws.ev[2]));
        SCG_CUDA(cudaEventElapsedTime(&b, h->ws.ev[2], h->ws.ev[3]));
        if (rep > 0 && a + b < t) t = a + b;
    }
    *ms = t;
    return SCG_OK;
}

int scg_autotune_ex(scg_index *h, const scg_search_params *p, const float *dQ, int nq, int *d_ids, float *d_dists,
                    int *d_sums, float min_agree, scg_tune_record *rec) {
    int rc;
    if ((rc = check_ready(h))) return rc;
    if ((rc = check_params(h, p, nq))) return rc;
    if (nq < 1 || !dQ || !d_ids || !d_dists || !d_sums || !rec) return fail(SCG_ERR_ARG, "autotune needs a batch and a record");
    if (!(min_agree >= 0.0f && min_agree <= 1.0f)) return fail(SCG_ERR_ARG, "min_agree must be in [0, 1]");
    std::lock_guard<std::mutex> g(h->mu);
    if ((rc = set_device(h))) return rc;
    memset(rec, 0, sizeof(*rec));
    const int form = scan_form(p->precision) == SCG_FAST ? 1 : 0;
    const int saved_upl = h->tuned_upl[form], saved_prefix = h->prefix_len;
    const bool saved_split = h->split;
    auto restore = [&]() {
        h->tuned_upl[form] = saved_upl;
        h->prefix_len = saved_prefix;
        h->split = saved_split;
    };
    // (1) candidates per lane of the scan
    const int ucand[3] = {2, 4, 8};
    float best = 3.4e38f;
    for (int i = 0; i < 3; i++) {
        h->tuned_upl[form] = ucand[i];
        if ((rc = tune_time(h, p, dQ, nq, d_ids, d_dists, d_sums, 3, &rec->upl_ms[i]))) { restore(); return rc; }
        if (rec->upl_ms[i] < best) {
            best = rec->upl_ms[i];
            rec->upl = ucand[i];
        }
    }
    h->tuned_upl[form] = rec->upl;
    // (2) the sorted coarse-prefix length (0: the density rule); results do
    // not depend on it, a short prefix only sends queries to a complete sort
    const int pcand[4] = {0, 128, 256, 512};
    best = 3.4e38f;
    for (int i = 0; i < 4; i++) {
        h->prefix_len = pcand[i];
        if ((rc = tune_time(h, p, dQ, nq, d_ids, d_dists, d_sums, 3, &rec->prefix_ms[i]))) { restore(); return rc; }
        if (rec->prefix_ms[i] < best) {
            best = rec->prefix_ms[i];
            rec->prefix = pcand[i];
        }
    }
    h->prefix_len = rec->prefix;
    // (3) kernel organisation: split selection + scan, or the fused kernel.
    // A split run whose visited lists outgrew the pool is searched again by
    // the fused kernel, and its events then time only that second search:
    // such a split never wins (it costs its own kernels on top).
    best = 3.4e38f;
    for (int i = 0; i < 2; i++) {
        h->split = i == 0;
        if ((rc = tune_time(h, p, dQ, nq, d_ids, d_dists, d_sums, 3, &rec->split_ms[i]))) { restore(); return rc; }
        const bool fell_back = i == 0 && !h->ws.last_split;
        if (!fell_back && rec->split_ms[i] < best) {
            best = rec->split_ms[i];
            rec->split = i == 0 ? 1 : 0;
        }
    }
    h->split = rec->split != 0;
    // (4) the re-rank shortlist: the fastest length whose top-R ids agree
    // with the caller's length on at least min_agree of the queries
    if (p->rerank > 0) {
        const int R = p->R;
        std::vector<int> ref((size_t)nq * R), got((size_t)nq * R);
        if ((rc = run_search(h, &h->ws, nullptr, p, dQ, nq, d_ids, d_dists, d_sums, h->stream, true))) {
            restore();
            return rc;
        }
        SCG_CUDA(cudaMemcpy(ref.data(), d_ids, sizeof(int) * ref.size(), cudaMemcpyDeviceToHost));
        best = 3.4e38f;
        for (int i = 0, L = R; i < 5 && L <= 1024; i++, L *= 2) {
            scg_search_params q = *p;
            q.rerank = L;
            rec->shortlist_L[i] = L;
            if ((rc = tune_time(h, &q, dQ, nq, d_ids, d_dists, d_sums, 3, &rec->shortlist_ms[i]))) {
                restore();
                return rc;
            }
            SCG_CUDA(cudaMemcpy(got.data(), d_ids, sizeof(int) * got.size(), cudaMemcpyDeviceToHost));
            int same = 0;
            for (int qi = 0; qi < nq; qi++) {
                std::vector<int> x(ref.begin() + (size_t)qi * R, ref.begin() + (size_t)(qi + 1) * R);
                std::vector<int> y(got.begin() + (size_t)qi * R, got.begin() + (size_t)(qi + 1) * R);
                std::sort(x.begin(), x.end());
                std::sort(y.begin(), y.end());
                same += x == y ? 1 : 0;
            }
            rec->shortlist_agree[i] = (float)same / (float)nq;
            if (rec->shortlist_agree[i] >= min_agree && rec->shortlist_ms[i] < best) {
                best = rec->shortlist_ms[i];
                rec->shortlist = L;
            }
        }
        if (rec->shortlist == 0) rec->shortlist = p->rerank;
    }
    return SCG_OK;
}

int scg_set_kernel_split(scg_index *h, int on) {
    if (!h) return fail(SCG_ERR_ARG, "null index");
    std::lock_guard<std::mutex> g(h->mu);
    h->split = on != 0;
    return SCG_OK;
}

int scg_set_rank_limit(scg_index *h, int M) {
    if (!h) return fail(SCG_ERR_ARG, "null index");
    if (M < 0) return fail(SCG_ERR_ARG, "rank limit must be >= 0");
    std::lock_guard<std::mutex> g(h->mu);
    h->rank_limit = M;
    return SCG_OK;
}

int scg_set_query_targets(scg_index *h, const int *d_T) {
    if (!h) return fail(SCG_ERR_ARG, "null index");
    h->d_Tq = d_T;
    return SCG_OK;
}

int scg_set_cell_budget(scg_index *h, int max_cells) {
    if (!h) return fail(SCG_ERR_ARG, "null index");
    if (max_cells < 64) return fail(SCG_ERR_ARG, "cell budget must be >= 64");
    h->cap_rec = max_cells;
    return SCG_OK;
}

// Codes through tensor-core distance tables and exact re-checks
// (encode_tc.cu), a chunk of rows at a time: IVF/IMI (nc = 0) or the second
// candidate's nc nearest coarse centroids with float-rounded comparisons.
static int encode_tc(scg_index *h, const float *dX, int64_t n, int nc, uint16_t *d_cid, uint8_t *d_codes,
                     cudaStream_t s) {
    int rc;
    const int bsc = h->dim / h->mc, bsp = h->dim / h->mp;
    if (!h->enc_ready) {
        if ((rc = h->enc_nc.ensure(4ull * h->mc * h->kc))) return rc;
        if ((rc = h->enc_nr.ensure(4ull * h->mp * h->kp))) return rc;
        if ((rc = h->enc_cmax.ensure(4ull * h->mc))) return rc;
        if ((rc = h->enc_rmax.ensure(4ull * h->mp))) return rc;
        launch_norms(h->cq.as<float>(), h->mc * h->kc, bsc, h->enc_nc.as<float>(), s);
        launch_norms(h->pq.as<float>(), h->mp * h->kp, bsp, h->enc_nr.as<float>(), s);
        launch_segmax(h->enc_nc.as<float>(), h->mc, h->kc, h->enc_cmax.as<float>(), s);
        launch_segmax(h->enc_nr.as<float>(), h->mp, h->kp, h->enc_rmax.as<float>(), s);
        SCG_CUDA(cudaGetLastError());
        h->enc_ready = true;
    }
    const int64_t RC = 32768;
    const int64_t width = std::max<int64_t>((int64_t)h->mc * h->kc, (int64_t)h->mp * h->kp);
    if ((rc = h->enc_tab.ensure(4ull * RC * width))) return rc;
    if ((rc = h->enc_res.ensure(4ull * RC * h->dim))) return rc;
    if ((rc = h->enc_status.ensure(16))) return rc;
    SCG_CUDA(cudaMemsetAsync(h->enc_status.p, 0, 16, s));
    for (int64_t r0 = 0; r0 < n; r0 += RC) {
        const int nr = (int)std::min<int64_t>(RC, n - r0);
        TablesArgs ta;
        memset(&ta, 0, sizeof(ta));
        ta.dim = h->dim; ta.mc = h->mc; ta.kc = h->kc; ta.mp = h->mp; ta.kp = h->kp; ta.nq = nr;
        ta.Q = dX + (size_t)r0 * h->dim;
        ta.cq = h->cq.as<float>(); ta.pq = h->pq.as<float>();
        ta.norm_c = h->enc_nc.as<float>(); ta.norm_r = h->enc_nr.as<float>();
        ta.dqc = h->enc_tab.as<float>(); ta.dqr = h->enc_tab.as<float>();
        ta.status = h->enc_status.as<int>();
        ta.segs = 1;
        launch_tables_tc(ta, 3, 1, s);
        PickArgs pa;
        pa.X = ta.Q; pa.n = nr; pa.dim = h->dim; pa.nseg = h->mc; pa.kseg = h->kc; pa.len = bsc;
        pa.C = h->cq.as<float>(); pa.tab = h->enc_tab.as<float>(); pa.segmax = h->enc_cmax.as<float>();
        pa.cid = d_cid + (size_t)r0 * (nc ? nc : h->mc); pa.code = nullptr; pa.resid = h->enc_res.as<float>();
        pa.status = h->enc_status.as<int>();
        pa.nbest = nc ? nc : 1;
        pa.fcmp = nc ? 1 : 0;
        launch_pick(pa, s);
        ta.Q = h->enc_res.as<float>();
        ta.segs = 2;
        launch_tables_tc(ta, 3, 1, s);
        pa.X = h->enc_res.as<float>(); pa.nseg = h->mp; pa.kseg = h->kp; pa.len = bsp;
        pa.C = h->pq.as<float>(); pa.segmax = h->enc_rmax.as<float>();
        pa.cid = nullptr; pa.code = d_codes + (size_t)r0 * h->mp; pa.resid = nullptr;
        pa.nbest = 1;
        launch_pick(pa, s);
        SCG_CUDA(cudaGetLastError());
    }
    int st = 0;
    SCG_CUDA(cudaMemcpyAsync(&st, h->enc_status.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    SCG_CUDA(cudaStreamSynchronize(s));
    if (st & ST_TC_TIMEOUT) return fail(SCG_ERR_CUDA, "a tensor-core distance tile did not complete in time");
    if (st & ST_BAD_ARG) return fail(SCG_ERR_ARG, "a row has no finite distance (NaN or infinite input)");
    return SCG_OK;
}

int scg_build_index(scg_index *h, const float *dX, int64_t n, int nc, void *stream) {
    if (!h) return fail(SCG_ERR_ARG, "null index");
    if (!h->have_codebooks) return fail(SCG_ERR_STATE, "load codebooks first");
    if (n < 0 || n > 0xfffffffeLL) return fail(SCG_ERR_ARG, "n out of range");
    if (n > 0 && !dX) return fail(SCG_ERR_ARG, "null buffer");
    if (nc != 0 && nc != 2 && nc != 3) return fail(SCG_ERR_ARG, "nc must be 0 (IVF/IMI), 2 or 3 (second candidate)");
    if (nc && h->mc != 1) return fail(SCG_ERR_ARG, "the second-candidate index needs mc = 1");
    const int parts = nc ? nc : h->mc;
    const int64_t ncells = ipow(h->kc, parts);
    if (ncells >= (1ll << 32)) return fail(SCG_ERR_ARG, "too many cells");
    int rc;
    DevBuf cid, codes, work;
    if ((rc = cid.ensure(2ull * (n ? n : 1) * parts))) return rc;
    if ((rc = codes.ensure((size_t)(n ? n : 1) * h->mp))) { cid.release(); return rc; }
    auto release = [&]() { cid.release(); codes.release(); work.release(); };
    if (n > 0 && (rc = scg_encode_device(h, dX, n, nc, cid.as<uint16_t>(), codes.as<uint8_t>(), stream))) {
        release();
        return rc;
    }
    std::lock_guard<std::mutex> g(h->mu);
    if ((rc = set_device(h))) { release(); return rc; }
    cudaStream_t s = stream ? (cudaStream_t)stream : h->stream;
    if ((rc = work.ensure(build_work_bytes(n, ncells))) ||
        (rc = h->off.ensure(4ull * (ncells + 1))) || (rc = h->pid.ensure(4ull * (n ? n : 1))) ||
        (rc = h->codes.ensure((size_t)(n ? n : 1) * h->mp))) {
        release();
        return rc;
    }
    if (n > 0) {
        launch_build_csr(cid.as<uint16_t>(), codes.as<uint8_t>(), n, parts, h->kc, h->mp, ncells,
                         work.as<unsigned char>(), h->off.as<uint32_t>(), h->pid.as<int>(), h->codes.as<uint8_t>(), s);
    } else {
        SCG_CUDA(cudaMemsetAsync(h->off.p, 0, 4ull * (ncells + 1), s));
    }
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    release();
    if (e != cudaSuccess) return cuda_fail(e, "scg_build_index");
    h->N = n;
    h->ncells = ncells;
    h->have_csr = true;
    if (h->dens.p) SCG_CUDA(cudaMemset(h->dens.p, 0, 16));
    h->have_vterm = false;
    return SCG_OK;
}

int scg_write_edat(scg_index *h, const char *path) {
    if (!h || !path) return fail(SCG_ERR_ARG, "null argument");
    if (!h->have_csr) return fail(SCG_ERR_STATE, "encoded data not loaded");
    std::lock_guard<std::mutex> g(h->mu);
    int rc;
    if ((rc = set_device(h))) return rc;
    const int64_t nc = h->ncells, N = h->N;
    std::vector<uint32_t> off((size_t)nc + 1);
    std::vector<int> pid((size_t)(N ? N : 1));
    std::vector<uint8_t> codes((size_t)(N ? N : 1) * h->mp);
    SCG_CUDA(cudaMemcpy(off.data(), h->off.p, 4ull * (nc + 1), cudaMemcpyDeviceToHost));
    if (N) {
        SCG_CUDA(cudaMemcpy(pid.data(), h->pid.p, 4ull * N, cudaMemcpyDeviceToHost));
        SCG_CUDA(cudaMemcpy(codes.data(), h->codes.p, (size_t)N * h->mp, cudaMemcpyDeviceToHost));
    }
    std::ofstream f(path, std::ios::binary | std::ios::trunc);
    if (!f) return fail(SCG_ERR_IO, std::string("cannot write ") + path);
    int non_empty = 0;
    for (int64_t c = 0; c < nc; c++) non_empty += off[(size_t)c + 1] > off[(size_t)c];
    const int hdr[2] = {non_empty, (int)N};
    std::vector<char> buf;
    buf.reserve(64 << 20);
    auto put = [&](const void *p, size_t bytes) {
        const char *q = (const char *)p;
        buf.insert(buf.end(), q, q + bytes);
        if (buf.size() >= (64u << 20)) {
            f.write(buf.data(), (std::streamsize)buf.size());
            buf.clear();
        }
    };
    put(hdr, sizeof(hdr));
    for (int64_t c = 0; c < nc; c++) {
        const uint32_t a = off[(size_t)c], b = off[(size_t)c + 1];
        const int l = (int)(b - a);
        put(&l, 4);
        if (l) {
            put(pid.data() + a, 4ull * l);
            put(codes.data() + (size_t)a * h->mp, (size_t)l * h->mp);
        }
    }
    f.write(buf.data(), (std::streamsize)buf.size());
    if (!f) return fail(SCG_ERR_IO, std::string("short write to ") + path);
    return SCG_OK;
}

int scg_train_codebooks(const float *dX, int64_t n, int dim, int mc, int kc, int mp, int kp, int iters,
                        uint64_t seed, float *d_cq, float *d_pq, int device, void *stream) {
    if (!dX || !d_cq || !d_pq) return fail(SCG_ERR_ARG, "null buffer");
    if (n < 1 || dim < 1 || mc < 1 || kc < 1 || mp < 1 || kp < 1 || iters < 0)
        return fail(SCG_ERR_ARG, "non-positive shape");
    if (dim % mc || dim % mp) return fail(SCG_ERR_ARG, "dim must divide by mc and mp");
    if ((kc > 1 && n < kc) || n < kp) return fail(SCG_ERR_ARG, "fewer training rows than centroids");
    if (kc > 65535 || kp > 256) return fail(SCG_ERR_ARG, "kc must be < 65536 and kp <= 256");
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t budget = 1ll << 28;  // floats of distance table per row chunk
    auto chunk_of = [&](int nseg, int k) { return std::max<int64_t>(128, std::min<int64_t>(n, budget / ((int64_t)nseg * k))); };
    const int64_t ch_c = chunk_of(mc, kc), ch_p = chunk_of(mp, kp);
    const size_t wbytes = std::max(kmeans_work_bytes(n, mc, kc, dim / mc, ch_c), kmeans_work_bytes(n, mp, kp, dim / mp, ch_p));
    DevBuf work, resid, asg, status;
    int rc;
    if ((rc = work.ensure(wbytes))) return rc;
    if ((rc = resid.ensure(4ull * n * dim))) { work.release(); return rc; }
    if ((rc = asg.ensure(4ull * n * mc))) { work.release(); resid.release(); return rc; }
    if ((rc = status.ensure(16))) { work.release(); resid.release(); asg.release(); return rc; }
    auto release = [&]() { work.release(); resid.release(); asg.release(); status.release(); };
    if ((e = cudaMemsetAsync(status.p, 0, 16, s)) != cudaSuccess) { release(); return cuda_fail(e, "memset"); }
    // coarse codebook (kc == 1: the zero centroid of plain PQ) and residuals
    if (kc == 1) {
        e = cudaMemsetAsync(d_cq, 0, 4ull * dim, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(resid.p, dX, 4ull * n * dim, cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) { release(); return cuda_fail(e, "zero coarse centroid"); }
    } else {
        rc = kmeans_segments(dX, n, dim, mc, kc, iters, seed, d_cq, work.as<unsigned char>(), ch_c, status.as<int>(),
                             asg.as<int>(), s);
        if (rc) { release(); return rc; }
        launch_residual(dX, n, dim, mc, kc, d_cq, asg.as<int>(), resid.as<float>(), s);
    }
    // residual PQ codebooks
    rc = kmeans_segments(resid.as<float>(), n, dim, mp, kp, iters, seed ^ 0x5851f42d4c957f2dull, d_pq,
                         work.as<unsigned char>(), ch_p, status.as<int>(), nullptr, s);
    if (rc) { release(); return rc; }
    int st = 0;
    e = cudaMemcpyAsync(&st, status.p, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    release();
    if (e != cudaSuccess) return cuda_fail(e, "scg_train_codebooks");
    if (st) return status_result(st);
    return SCG_OK;
}

int scg_kmeans(const float *X, int64_t n, int dim, int nseg, int k, int iters, uint64_t seed, float *centers,
               int *labels, int device) {
    if (!X || !centers) return fail(SCG_ERR_ARG, "null buffer");
    if (n < 1 || dim < 1 || nseg < 1 || k < 1 || iters < 0 || dim % nseg) return fail(SCG_ERR_ARG, "bad shape");
    if (n < k) return fail(SCG_ERR_ARG, "fewer rows than centroids");
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    const int64_t chunk = std::max<int64_t>(128, std::min<int64_t>(n, (1ll << 28) / ((int64_t)nseg * k)));
    DevBuf dx, dc, work, asg, status;
    int rc;
    auto release = [&]() { dx.release(); dc.release(); work.release(); asg.release(); status.release(); };
    if ((rc = dx.ensure(4ull * n * dim)) || (rc = dc.ensure(4ull * nseg * k * (dim / nseg))) ||
        (rc = work.ensure(kmeans_work_bytes(n, nseg, k, dim / nseg, chunk))) || (rc = asg.ensure(4ull * nseg * n)) ||
        (rc = status.ensure(16))) {
        release();
        return rc;
    }
    e = cudaMemcpy(dx.p, X, 4ull * n * dim, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(status.p, 0, 16);
    if (e != cudaSuccess) { release(); return cuda_fail(e, "scg_kmeans copies"); }
    rc = kmeans_segments(dx.as<float>(), n, dim, nseg, k, iters, seed, dc.as<float>(), work.as<unsigned char>(), chunk,
                         status.as<int>(), asg.as<int>(), nullptr);
    int st = 0;
    if (rc == SCG_OK) {
        e = cudaMemcpy(centers, dc.p, 4ull * nseg * k * (dim / nseg), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess && labels) e = cudaMemcpy(labels, asg.p, 4ull * nseg * n, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(&st, status.p, sizeof(int), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) rc = cuda_fail(e, "scg_kmeans results");
    }
    release();
    if (rc) return rc;
    return st ? status_result(st) : SCG_OK;
}

int scg_exact_nn(const float *dX, int64_t n, const float *dQ, int nq, int dim, int *d_ids, float *d_dists,
                 int device, void *stream) {
    if (!dX || !dQ || !d_ids) return fail(SCG_ERR_ARG, "null buffer");
    if (n < 1 || nq < 1 || dim < 1) return fail(SCG_ERR_ARG, "non-positive shape");
    if (n > 0x7fffffffll) return fail(SCG_ERR_ARG, "row indices must fit int32");
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    cudaStream_t s = (cudaStream_t)stream;
    // distance tables of at most 2^28 floats per chunk of rows
    const int64_t chunk = std::max<int64_t>(256, std::min<int64_t>(n, (1ll << 28) / nq));
    DevBuf work, status;
    int rc;
    if ((rc = work.ensure(exact_nn_work_bytes(nq, chunk)))) return rc;
    if ((rc = status.ensure(16))) { work.release(); return rc; }
    auto release = [&]() { work.release(); status.release(); };
    if ((e = cudaMemsetAsync(status.p, 0, 16, s)) != cudaSuccess) { release(); return cuda_fail(e, "memset"); }
    rc = exact_nn(dX, n, dQ, nq, dim, d_ids, d_dists, work.as<unsigned char>(), chunk, status.as<int>(), s);
    int st = 0;
    e = cudaMemcpyAsync(&st, status.p, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    release();
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_fail(e, "scg_exact_nn");
    return st ? status_result(st) : SCG_OK;
}

int scg_set_encoder(scg_index *h, int method) {
    if (!h) return fail(SCG_ERR_ARG, "null index");
    if (method != SCG_ENC_EXACT && method != SCG_ENC_TENSOR) return fail(SCG_ERR_ARG, "unknown encoder");
    std::lock_guard<std::mutex> g(h->mu);
    h->encoder = method;
    return SCG_OK;
}

int scg_encode_device(scg_index *h, const float *dX, int64_t n, int nc, uint16_t *d_cid, uint8_t *d_codes,
                      void *stream) {
    if (!h) return fail(SCG_ERR_ARG, "null index");
    if (!h->have_codebooks) return fail(SCG_ERR_STATE, "codebooks not loaded");
    if (n < 0) return fail(SCG_ERR_ARG, "n < 0");
    if (n > 0 && (!dX || !d_cid || !d_codes)) return fail(SCG_ERR_ARG, "null buffer");
    if (nc != 0 && nc != 2 && nc != 3) return fail(SCG_ERR_ARG, "nc must be 0 (IVF/IMI), 2 or 3");
    if (nc && h->mc != 1) return fail(SCG_ERR_ARG, "the second-candidate encoder needs mc = 1");
    if (nc > h->kc) return fail(SCG_ERR_ARG, "nc > kc");
    int mcp = nc ? 1 : h->mc;
    std::lock_guard<std::mutex> g(h->mu);
    int rc;
    if ((rc = set_device(h))) return rc;
    cudaStream_t s = stream ? (cudaStream_t)stream : h->stream;
    if (h->encoder == SCG_ENC_TENSOR) return n > 0 ? encode_tc(h, dX, n, nc, d_cid, d_codes, s) : SCG_OK;
    if (encode_smem_bytes(h->dim, mcp) > 227 * 1024)
        return fail(SCG_ERR_ARG, "dimension too large for the exact encoder's shared-memory tile");
    EncodeArgs a;
    a.dim = h->dim; a.mc = h->mc; a.kc = h->kc; a.mp = h->mp; a.kp = h->kp; a.nc = nc; a.n = n;
    a.X = dX; a.cq = h->cq.as<float>(); a.pq = h->pq.as<float>(); a.cid = d_cid; a.codes = d_codes;
    launch_encode(a, s);
    SCG_CUDA(cudaGetLastError());
    SCG_CUDA(cudaStreamSynchronize(s));
    return SCG_OK;
}

static int encode_host(scg_index *h, const float *X, int64_t n, int nc, uint16_t *cid, uint8_t *codes) {
    if (!h) return fail(SCG_ERR_ARG, "null index");
    if (!h->have_codebooks) return fail(SCG_ERR_STATE, "codebooks not loaded");
    if (n <= 0) return n == 0 ? SCG_OK : fail(SCG_ERR_ARG, "n < 0");
    if (!X || !cid || !codes) return fail(SCG_ERR_ARG, "null buffer");
    int rc;
    if ((rc = set_device(h))) return rc;
    int ncid = nc ? nc : h->mc;
    DevBuf x, c, k;
    if ((rc = x.ensure(sizeof(float) * (size_t)n * h->dim))) return rc;
    if ((rc = c.ensure(sizeof(uint16_t) * (size_t)n * ncid))) { x.release(); return rc; }
    if ((rc = k.ensure((size_t)n * h->mp))) { x.release(); c.release(); return rc; }
    cudaError_t e = copy_in(x.p, X, sizeof(float) * (size_t)n * h->dim, h->stream);
    if (e == cudaSuccess) {
        rc = scg_encode_device(h, x.as<float>(), n, nc, c.as<uint16_t>(), k.as<uint8_t>(), nullptr);
        if (rc == SCG_OK) {
            e = cudaMemcpy(cid, c.p, sizeof(uint16_t) * (size_t)n * ncid, cudaMemcpyDeviceToHost);
            if (e == cudaSuccess) e = cudaMemcpy(codes, k.p, (size_t)n * h->mp, cudaMemcpyDeviceToHost);
        }
    }
    x.release(); c.release(); k.release();
    if (e != cudaSuccess) return cuda_fail(e, "encode copies");
    return rc;
}

int scg_encode(scg_index *h, const float *X, int64_t n, uint16_t *cid, uint8_t *codes) {
    return encode_host(h, X, n, 0, cid, codes);
}

int scg_sc_encode(scg_index *h, const float *X, int64_t n, int nc, uint16_t *cid, uint8_t *codes) {
    if (nc < 2) return fail(SCG_ERR_ARG, "nc must be >= 2");
    return encode_host(h, X, n, nc, cid, codes);
}

int scg_last_query_stats(scg_index *h, int *nvis, int *empty, int nq) {
    if (!h) return fail(SCG_ERR_ARG, "null index");
    if (nq < 0 || nq > h->ws.last_nq) return fail(SCG_ERR_ARG, "nq exceeds the last search's batch");
    std::lock_guard<std::mutex> g(h->mu);
    int rc;
    if ((rc = set_device(h))) return rc;
    if (nvis && nq) SCG_CUDA(cudaMemcpy(nvis, h->ws.nvis.p, sizeof(int) * (size_t)nq, cudaMemcpyDeviceToHost));
    if (empty && nq) SCG_CUDA(cudaMemcpy(empty, h->ws.empty.p, sizeof(int) * (size_t)nq, cudaMemcpyDeviceToHost));
    return SCG_OK;
}

int scg_last_timings(scg_index *h, float *ms, int n) {
    if (!h || !ms) return fail(SCG_ERR_ARG, "null argument");
    if (h->ws.last_nq <= 0) return fail(SCG_ERR_STATE, "no search has run");
    std::lock_guard<std::mutex> g(h->mu);
    int rc;
    if ((rc = set_device(h))) return rc;
    float t[5] = {0, 0, 0, 0, 0};
    SCG_CUDA(cudaEventElapsedTime(&t[0], h->ws.ev[0], h->ws.ev[1]));
    SCG_CUDA(cudaEventElapsedTime(&t[1], h->ws.ev[1], h->ws.ev[2]));
    SCG_CUDA(cudaEventElapsedTime(&t[2], h->ws.ev[2], h->ws.ev[3]));
    if (h->ws.last_split) {
        SCG_CUDA(cudaEventElapsedTime(&t[3], h->ws.ev[1], h->ws.ev[4]));
        SCG_CUDA(cudaEventElapsedTime(&t[4], h->ws.ev[4], h->ws.ev[2]));
    }
    for (int i = 0; i < n && i < 5; i++) ms[i] = t[i];
    return SCG_OK;
}

int scg_last_launches(scg_index *h, int *count) {
    if (!h || !count) return fail(SCG_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> g(h->mu);
    if (h->ws.last_nq <= 0) return fail(SCG_ERR_STATE, "no search has run");
    *count = h->ws.last_launches;
    return SCG_OK;
}

int scg_cell_counts(scg_index *h, int *L, int64_t ncells) {
    if (!h || !L) return fail(SCG_ERR_ARG, "null argument");
    if (!h->have_csr) return fail(SCG_ERR_STATE, "encoded data not loaded");
    if (ncells != h->ncells) return fail(SCG_ERR_ARG, "ncells differs from the loaded index");
    std::lock_guard<std::mutex> g(h->mu);
    int rc;
    if ((rc = set_device(h))) return rc;
    SCG_CUDA(cudaMemcpy(L, h->off.as<uint32_t>() + 1, sizeof(int) * (size_t)ncells, cudaMemcpyDeviceToHost));
    return SCG_OK;
}

int scg_set_phase_counters(scg_index *h, int on) {
    if (!h) return fail(SCG_ERR_ARG, "null index");
    h->ws.phase_on = on != 0;
    return SCG_OK;
}

int scg_last_phase_counters(scg_index *h, long long *out, int n) {
    if (!h || !out) return fail(SCG_ERR_ARG, "null argument");
    if (!h->ws.phase_on || !h->ws.phase.p) return fail(SCG_ERR_STATE, "phase counters are off");
    std::lock_guard<std::mutex> g(h->mu);
    int rc;
    if ((rc = set_device(h))) return rc;
    long long tmp[16];
    SCG_CUDA(cudaMemcpy(tmp, h->ws.phase.p, sizeof(tmp), cudaMemcpyDeviceToHost));
    for (int i = 0; i < n && i < 16; i++) out[i] = tmp[i];
    return SCG_OK;
}

int scg_index_info(scg_index *h, int *dim, int *mc, int *kc, int *mp, int *kp, int64_t *N) {
    if (!h) return fail(SCG_ERR_ARG, "null index");
    if (dim) *dim = h->dim;
    if (mc) *mc = h->mc;
    if (kc) *kc = h->kc;
    if (mp) *mp = h->mp;
    if (kp) *kp = h->kp;
    if (N) *N = h->N;
    return SCG_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Search without allocation.
//
// Some callers cannot allocate device memory at search time -- code running
// under a memory pool that forbids cudaMalloc, callers that must not change
// the device's allocation state while other work runs, or processes whose
// allocator is owned by someone else.  scg_search_device_noalloc serves them
// from one file-scope device array of SCG_NOALLOC_SCRATCH_BYTES, which every
// GPU that loads this library holds until the process exits.

namespace {

constexpr size_t SCG_NOALLOC_SCRATCH_BYTES = 48ull << 20;  // 48 MiB
constexpr int NOALLOC_CELLS = 8192;                        // cells per query (budget)
constexpr int NOALLOC_SURVIVORS = 8192;                    // scan survivors per query

}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[SCG_NOALLOC_SCRATCH_BYTES];

namespace {

std::mutex g_noalloc_mu;
void *g_noalloc_ptr[64] = {nullptr};

// Device address of the scratch array on the current device (the host-side
// name of the array is only a stand-in).  Looked up once per device.
int noalloc_scratch(int device, unsigned char **out) {
    if (device < 0 || device >= 64) return fail(SCG_ERR_ARG, "device index out of range");
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    if (!g_noalloc_ptr[device]) {
        void *ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(scratch)");
        g_noalloc_ptr[device] = ptr;
    }
    *out = (unsigned char *)g_noalloc_ptr[device];
    return SCG_OK;
}

size_t up256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

extern "C" int scg_search_device_noalloc(scg_index *h, const scg_search_params *p, const float *dQ, int nq,
                                         int *d_ids, float *d_dists, int *d_sums, void *stream) {
    int rc;
    if ((rc = check_ready(h))) return rc;
    if ((rc = check_params(h, p, nq))) return rc;
    if (nq > 0 && (!dQ || !d_ids || !d_dists || !d_sums)) return fail(SCG_ERR_ARG, "null buffer");
    if (p->rerank != 0) return fail(SCG_ERR_ARG, "the allocation-free search does not re-rank (rerank must be 0)");
    std::lock_guard<std::mutex> g(h->mu);
    // read under the lock: every builder of the per-vector term holds it and
    // synchronises its stream before setting the flag, so a set flag means
    // the term is complete in device memory before this call enqueues work
    if (scan_form(p->precision) == SCG_FAST && !h->have_vterm)
        return fail(SCG_ERR_STATE,
                    "the per-vector term of the tensor-core forms is built by their first call of scg_search or "
                    "scg_search_device; make one before searching without allocation");
    if ((rc = set_device(h))) return rc;
    if (nq == 0) return SCG_OK;
    unsigned char *base = nullptr;
    if ((rc = noalloc_scratch(h->device, &base))) return rc;
    cudaStream_t s = stream ? (cudaStream_t)stream : h->stream;

    // carve the scratch: per-query tables first, then per-CTA slots
    const size_t per_query = up256(sizeof(float) * (size_t)h->mc * h->kc) + up256(sizeof(float) * (size_t)h->mp * h->kp);
    const size_t slot_bytes = up256(4ull * NOALLOC_CELLS) * 3 + up256(4ull * (NOALLOC_CELLS + 1)) * 2 +
                              up256(8ull * NOALLOC_SURVIVORS);
    // bytes n queries need besides the per-CTA slots: qn, qsum, nvis, empty,
    // the status word and the counter, and the per-query tables
    auto fixed_of = [&](size_t n) { return 4 * up256(sizeof(float) * n * 2) + 2 * 256 + per_query * n; };
    const int upl = h->tuned_upl[scan_form(p->precision) == SCG_FAST ? 1 : 0];
    const int rot = search_rot_form(scan_form(p->precision), h->mp, h->kp) ? 1 : 0;
    int per_sm = search_max_blocks_per_sm(p->mode, h->kc, h->mp, h->kp, upl, 0, rot);
    if (per_sm < 1) return fail(SCG_ERR_ARG, "search kernel does not fit on an SM for this shape");
    int grid = h->num_sms * per_sm;
    if (grid > nq) grid = nq;
    if (fixed_of((size_t)nq) + slot_bytes > SCG_NOALLOC_SCRATCH_BYTES) {
        // the largest batch the same rule admits (one search slot at least)
        size_t lo = 0, hi = SCG_NOALLOC_SCRATCH_BYTES / per_query + 1;
        while (lo < hi) {
            const size_t mid = (lo + hi + 1) / 2;
            if (fixed_of(mid) + slot_bytes <= SCG_NOALLOC_SCRATCH_BYTES) lo = mid;
            else hi = mid - 1;
        }
        return fail(SCG_ERR_CAP, "nq = " + std::to_string(nq) + " exceeds the 48 MiB scratch of the allocation-free "
                    "search for this index (at most " + std::to_string(lo) + " queries per call)");
    }
    const size_t left = SCG_NOALLOC_SCRATCH_BYTES - fixed_of((size_t)nq);
    if ((size_t)grid * slot_bytes > left) grid = (int)(left / slot_bytes);
    if (grid < 1) return fail(SCG_ERR_CAP, "the allocation-free scratch has no room for a search slot");

    unsigned char *cur = base;
    auto take = [&](size_t bytes) {
        unsigned char *r = cur;
        cur += up256(bytes);
        return r;
    };
    float *dqc = (float *)take(sizeof(float) * (size_t)nq * h->mc * h->kc);
    float *dqr = (float *)take(sizeof(float) * (size_t)nq * h->mp * h->kp);
    float *qn = (float *)take(sizeof(float) * (size_t)nq * 2);
    float *qsum = (float *)take(sizeof(float) * (size_t)nq);
    int *nvis = (int *)take(sizeof(int) * (size_t)nq);
    int *empty = (int *)take(sizeof(int) * (size_t)nq);
    int *status = (int *)take(sizeof(int) * 4);
    int *counter = (int *)take(sizeof(int) * 4);
    uint32_t *rec_key = (uint32_t *)take(4ull * NOALLOC_CELLS * grid);
    uint32_t *rec_rank = (uint32_t *)take(4ull * NOALLOC_CELLS * grid);
    uint32_t *rec_cnt = (uint32_t *)take(4ull * NOALLOC_CELLS * grid);
    uint32_t *vis_cell = (uint32_t *)take(4ull * (NOALLOC_CELLS + 1) * grid);
    uint32_t *vis_pre = (uint32_t *)take(4ull * (NOALLOC_CELLS + 1) * grid);
    uint64_t *pend = (uint64_t *)take(8ull * NOALLOC_SURVIVORS * grid);
    if ((size_t)(cur - base) > SCG_NOALLOC_SCRATCH_BYTES) return fail(SCG_ERR_CAP, "allocation-free scratch overrun");

    TablesArgs ta;
    memset(&ta, 0, sizeof(ta));
    ta.dim = h->dim; ta.mc = h->mc; ta.kc = h->kc; ta.mp = h->mp; ta.kp = h->kp; ta.nq = nq;
    ta.Q = dQ;
    ta.cq = h->cq.as<float>(); ta.pq = h->pq.as<float>();
    ta.norm_c = h->norm_c.as<float>(); ta.norm_r = h->norm_r.as<float>();
    ta.dqc = dqc; ta.dqr = dqr; ta.qn = qn; ta.qsum = qsum;
    ta.lut_only = scan_form(p->precision) == SCG_FAST;
    ta.status = status;
    // the scratch keeps the previous call's contents: clear what starts at zero
    SCG_CUDA(cudaMemsetAsync(status, 0, sizeof(int) * 4, s));
    SCG_CUDA(cudaMemsetAsync(counter, 0, sizeof(int) * 4, s));
    launch_tables(ta, p->precision, s);
    SearchArgs sa;
    memset(&sa, 0, sizeof(sa));
    sa.mode = p->mode; sa.dim = h->dim; sa.mc = h->mc; sa.kc = h->kc; sa.mp = h->mp; sa.kp = h->kp;
    sa.nq = nq; sa.R = p->R; sa.w = p->w; sa.T = p->T; sa.precision = scan_form(p->precision);
    sa.rot = rot;
    sa.upl = upl;
    sa.Tq = h->d_Tq;
    sa.rank_limit = h->rank_limit;
    sa.dqc = dqc; sa.dqr = dqr; sa.qn = qn; sa.qsum = qsum;
    sa.off = h->off.as<uint32_t>(); sa.pid = h->pid.as<int>(); sa.codes = h->codes.as<uint8_t>();
    sa.dot_cr = h->dot_cr.as<float>();
    sa.vterm = h->vterm.as<float>();
    sa.ncells = (uint64_t)h->ncells;
    sa.N = h->N;
    sa.rec_key = rec_key; sa.rec_rank = rec_rank; sa.rec_cnt = rec_cnt;
    sa.vis_cell = vis_cell; sa.vis_pre = vis_pre;
    sa.cap_rec = NOALLOC_CELLS;
    sa.pend = pend;
    sa.pcap = NOALLOC_SURVIVORS;
    sa.qcounter = counter;
    sa.out_ids = d_ids; sa.out_d = d_dists; sa.out_sum = d_sums;
    sa.out_nvis = nvis; sa.out_empty = empty;
    sa.status = status;
    sa.phase_cycles = nullptr;
    if ((rc = search_launch(sa, 0, grid, s))) return rc;
    SCG_CUDA(cudaMemcpyAsync(h->ws.h_status, status, sizeof(int), cudaMemcpyDeviceToHost, s));
    SCG_CUDA(cudaStreamSynchronize(s));
    int st = *h->ws.h_status;
    if (st & ST_CELL_BUDGET)
        return fail(SCG_ERR_CAP, "a query needs more than the allocation-free search's 8192 cells or survivors");
    if (st & ST_TIE_OVERFLOW) return fail(SCG_ERR_CAP, "too many cells tie exactly at the cut key");
    if (st & ST_ITER_CAP) return fail(SCG_ERR_CAP, "cell selection did not converge within its round cap");
    if (st & ST_TC_TIMEOUT) return fail(SCG_ERR_CUDA, "a tensor-core table tile did not complete in time");
    if (st & ST_BAD_ARG) return fail(SCG_ERR_ARG, "the search kernel rejected its arguments");
    if (st) return fail(SCG_ERR_CUDA, "search kernel reported status " + std::to_string(st));
    return SCG_OK;
}
