/*
 * ref_harness.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * A thin C-callable driver around the reference library's OWN headers and
 * sources (compiled by oracle/Makefile from the reference tree into
 * oracle/_ref/libscref.so).  It exists so that tests can pin the C
 * restatement in sc_oracle.c against the reference itself, and so that
 * bench.py can time the reference's CPU search beside the GPU.
 *
 * The only change to the reference is the sequencing fix of query.h:167,179
 * (applied by the Makefile to a generated copy under oracle/_ref/): without
 * it the per-query tables are shifted by one slot and read uninitialised
 * memory.
 *
 * Parallel use follows the reference's own structure: the query classes are
 * not reentrant (pre_compute2 writes the members diff_qc/diff_qr), so each
 * OpenMP thread owns a clone that shares the index arrays and the
 * query-independent tables of a master object and owns only its per-query
 * tables and search scratch.
 */
#include <chrono>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "multi_query.h"
#include "sc_query.h"
#include "encoder.h"
#include "sc_encoder.h"
#include "evaluation.h"

using namespace SC;

namespace {

/* Gives access to the protected members of a reference query class. */
template <class Base>
struct Opened : public Base {
    Opened() : Base() {}
    explicit Opened(int nc) : Base(nc) {}
    void set_index(int dim, int mc, int kc, int mp, int kp, int N,
                   float *cq, float *pq, int *L, int *pid, unsigned char *codes, float *raw) {
        this->config.dim = dim; this->config.mc = mc; this->config.kc = kc;
        this->config.mp = mp; this->config.kp = kp; this->config.N = N;
        this->cq = cq; this->pq = pq; this->L = L; this->pid = pid; this->codes = codes;
        this->raw_data = raw;
        long s = 1;
        for (int i = 0; i < mc; i++) s *= kc;
        this->size = (int)s;
    }
    /* Shares the master's query-independent tables; owns its own per-query
     * tables (allocated like pre_compute1 does, query.h:95-96). */
    void share_tables(const Opened &m) {
        this->norm_c = m.norm_c; this->norm_r = m.norm_r; this->dot_cr = m.dot_cr;
        SimpleCluster::init_array(this->diff_qc, this->config.mc * this->config.kc);
        SimpleCluster::init_array(this->diff_qr, this->config.mp * this->config.kp);
    }
    float *get_norm_c() { return this->norm_c; }
    float *get_norm_r() { return this->norm_r; }
    float *get_dot_cr() { return this->dot_cr; }
    float *get_diff_qc() { return this->diff_qc; }
    float *get_diff_qr() { return this->diff_qr; }
    /* Drops the borrowed pointers so the reference destructor (query.cpp:37-61)
     * frees only what this object owns. */
    void release(bool owns_tables) {
        this->cq = nullptr; this->pq = nullptr; this->L = nullptr; this->pid = nullptr;
        this->codes = nullptr; this->raw_data = nullptr;
        if (!owns_tables) { this->norm_c = nullptr; this->norm_r = nullptr; this->dot_cr = nullptr; }
    }
};

typedef Opened<MultiQuery> OMulti;
typedef Opened<SCQuery> OSC;
/* SCQuery with three nearest centroids per cell (sc_query.cpp:21-25). */
struct OSC3 : public Opened<SCQuery> {
    OSC3() : Opened<SCQuery>(3) {}
};

struct Scratch {
    std::vector<float> v_tmp, q2;
    std::vector<int> tmp, hid1, hid2, hid3, hid4, hid5, hid6, s1, s2, prebuck, cache;
    std::vector<unsigned char> trav;
    /* mode 2: traversed[0] preset (test_sc_query.cpp:160-161); mode 3: the
     * kc^3 rank grid, nothing preset (the walk starts at (0, 0, 0)). */
    void init(int kc, int w, int mode) {
        v_tmp.assign((size_t)2 * kc + w, 0.0f);
        q2.assign(2, 0.0f);
        tmp.assign((size_t)2 * kc, 0);
        hid1.assign(w, 0); hid2.assign(w, 0); hid3.assign(w, 0); hid4.assign(w, 0);
        hid5.assign(w, 0); hid6.assign(w, 0);
        s1.assign(w, 0); s2.assign(w, 0); prebuck.assign(w, 0);
        /* the SC walks write cache[count2++] for every popped cell, empty ones
         * included, while w counts non-empty cells (sc_query.h:130,148,
         * 327,345): size it for the whole grid */
        const size_t grid = (size_t)kc * kc * (mode == 3 ? kc : 1);
        cache.assign(mode >= 2 ? grid + (size_t)w : (size_t)w, 0);
        trav.assign(grid, 0);
        if (mode == 2) trav[0] = 1;
    }
};

static MultiQuery *as_multi(OMulti &o) { return &o; }
static MultiQuery *as_multi(OSC &) { return nullptr; }
static MultiQuery *as_multi(OSC3 &) { return nullptr; }
static SCQuery *as_sc(OMulti &) { return nullptr; }
static SCQuery *as_sc(OSC &o) { return &o; }
static SCQuery *as_sc(OSC3 &o) { return &o; }

/* One query through the reference entry point for `mode`
 * (0 IVFADC query.h:202, 1 IMI multi_query.h:62, 2 SC sc_query.h:60).
 * Returns sum; result/dist are allocated by the reference. */
static int run_one(PQQuery &obj, MultiQuery *mq, SCQuery *sq, int mode, Scratch &s, float *q,
                   int R, int w, int T, int M, bool real_dist, int *&result, float *&dist,
                   int *empty) {
    int sum = 0;
    float *v_tmp = s.v_tmp.data(), *q2 = s.q2.data();
    int *hid1 = s.hid1.data(), *hid2 = s.hid2.data(), *hid3 = s.hid3.data(), *hid4 = s.hid4.data();
    int *s1 = s.s1.data(), *s2 = s.s2.data(), *prebuck = s.prebuck.data(), *cache = s.cache.data();
    bool *trav = reinterpret_cast<bool *>(s.trav.data());
    result = nullptr; dist = nullptr;
    if (mode == 0) {
        /* test_query.cpp:159-176: v_tmp, buckets and bk sized kc */
        obj.search_ivfadc(q, v_tmp, dist, result, hid1, prebuck, sum, R, w, T, real_dist, false);
    } else if (mode == 1 && mq) {
        int e = 0; double t1 = 0, t2 = 0;
        mq->search_multi2(q, v_tmp, dist, q2, s.tmp.data(), result,
                          hid1, hid2, hid3, hid4, s1, s2, prebuck, cache, trav,
                          sum, R, w, T, M, e, t1, t2, real_dist, false);
        if (empty) *empty = e;
    } else if (mode == 2 && sq) {
        sq->search_mr_ivf(q, v_tmp, dist, s.tmp.data(), result,
                          hid1, hid2, hid3, hid4, s1, s2, prebuck, cache, trav,
                          sum, R, w, T, M, real_dist, false);
    } else if (mode == 3 && sq) {
        int *hid5 = s.hid5.data(), *hid6 = s.hid6.data();
        sq->search_mr_ivf3(q, v_tmp, dist, s.tmp.data(), result,
                           hid1, hid2, hid3, hid4, hid5, hid6, s1, prebuck, cache, trav,
                           sum, R, w, T, M, real_dist, false);
    }
    return sum;
}

template <class Q>
int search_batch(int mode, int dim, int mc, int kc, int mp, int kp, int N,
                 float *cq, float *pq, int *L, int *pid, unsigned char *codes, float *raw,
                 const float *Qs, int nq, int R, int w, int T, const int *Tq, int M, int real_dist,
                 int nthreads, int *ids_out, float *dist_out, int *sum_out, double *seconds_out) {
    Q master;
    master.set_index(dim, mc, kc, mp, kp, N, cq, pq, L, pid, codes, raw);
    master.pre_compute1();
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    int nth = 1;
#ifdef _OPENMP
    nth = omp_get_max_threads();
#endif
    /* Clones and scratch are built before the clock starts. */
    std::vector<Q *> clones(nth);
    std::vector<Scratch> scratch(nth);
    int wcap = (mode == 0) ? (kc > w ? kc : w) : w;
    for (int t = 0; t < nth; t++) {
        clones[t] = new Q();
        clones[t]->set_index(dim, mc, kc, mp, kp, N, cq, pq, L, pid, codes, raw);
        clones[t]->share_tables(master);
        scratch[t].init(kc, wcap, mode);
    }
    auto t0 = std::chrono::steady_clock::now();
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 4)
#endif
    for (int i = 0; i < nq; i++) {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        std::vector<float> qv(Qs + (size_t)i * dim, Qs + (size_t)(i + 1) * dim);
        int *result; float *dist;
        int sum = run_one(*clones[tid], as_multi(*clones[tid]), as_sc(*clones[tid]), mode,
                          scratch[tid], qv.data(), R, w, Tq ? Tq[i] : T, M, real_dist != 0, result, dist,
                          nullptr);
        int m = sum < R ? sum : R;
        for (int j = 0; j < R; j++) {
            ids_out[(size_t)i * R + j] = j < m ? result[j] : -1;
            dist_out[(size_t)i * R + j] = j < m ? dist[j] : 0.0f;
        }
        sum_out[i] = sum;
        ::operator delete(result);
        ::operator delete(dist);
    }
    auto t1 = std::chrono::steady_clock::now();
    if (seconds_out) *seconds_out = std::chrono::duration<double>(t1 - t0).count();
    for (int t = 0; t < nth; t++) { clones[t]->release(false); delete clones[t]; }
    master.release(true);
    return 0;
}

} // namespace

extern "C" {

/* Runs nq queries through the reference search of `mode` with `nthreads`
 * OpenMP threads; writes the first min(R, sum) ids/distances the reference
 * returns per query (padding with -1) and each query's sum.  The wall time of
 * the query loop (pre_compute2 through top-R, steady_clock) goes to
 * *seconds_out. */
int ref_search_batch_ex(int mode, int dim, int mc, int kc, int mp, int kp, int N,
                        float *cq, float *pq, int *L, int *pid, unsigned char *codes, float *raw,
                        const float *Qs, int nq, int R, int w, int T, const int *Tq, int M, int real_dist,
                        int nthreads, int *ids_out, float *dist_out, int *sum_out, double *seconds_out);

int ref_search_batch(int mode, int dim, int mc, int kc, int mp, int kp, int N,
                     float *cq, float *pq, int *L, int *pid, unsigned char *codes, float *raw,
                     const float *Qs, int nq, int R, int w, int T, int real_dist, int nthreads,
                     int *ids_out, float *dist_out, int *sum_out, double *seconds_out) {
    return ref_search_batch_ex(mode, dim, mc, kc, mp, kp, N, cq, pq, L, pid, codes, raw, Qs, nq, R, w, T, nullptr, kc,
                               real_dist, nthreads, ids_out, dist_out, sum_out, seconds_out);
}

/* ref_search_batch with a per-query candidate target Tq[nq] (NULL: T for
 * every query; search_mr_ivf and search_multi2 take T per call,
 * sc_query.h:60-67, multi_query.h:62-70) and the coarse-list argument M of
 * search_multi2 / search_mr_ivf (kc in the reference's own tests). */
int ref_search_batch_ex(int mode, int dim, int mc, int kc, int mp, int kp, int N,
                        float *cq, float *pq, int *L, int *pid, unsigned char *codes, float *raw,
                        const float *Qs, int nq, int R, int w, int T, const int *Tq, int M, int real_dist,
                        int nthreads, int *ids_out, float *dist_out, int *sum_out, double *seconds_out) {
    if (mode == 2)
        return search_batch<OSC>(mode, dim, mc, kc, mp, kp, N, cq, pq, L, pid, codes, raw,
                                 Qs, nq, R, w, T, Tq, M, real_dist, nthreads, ids_out, dist_out, sum_out,
                                 seconds_out);
    if (mode == 3)
        return search_batch<OSC3>(mode, dim, mc, kc, mp, kp, N, cq, pq, L, pid, codes, raw,
                                  Qs, nq, R, w, T, Tq, M, real_dist, nthreads, ids_out, dist_out, sum_out,
                                  seconds_out);
    return search_batch<OMulti>(mode, dim, mc, kc, mp, kp, N, cq, pq, L, pid, codes, raw,
                                Qs, nq, R, w, T, Tq, M, real_dist, nthreads, ids_out, dist_out, sum_out,
                                seconds_out);
}

/* One query; copies all `sum` candidate (id, distance) pairs the reference
 * leaves in result/dist (permuted by its top-R step) when cap allows.
 * Returns sum, or -1 if cap is too small. */
int ref_search_one(int mode, int dim, int mc, int kc, int mp, int kp, int N,
                   float *cq, float *pq, int *L, int *pid, unsigned char *codes, float *raw,
                   const float *q, int R, int w, int T, int real_dist,
                   int *ids_all, float *dist_all, int cap, int *empty_out) {
    OMulti m1; OSC m2; OSC3 m3;
    Scratch s;
    int wcap = (mode == 0) ? (kc > w ? kc : w) : w;
    s.init(kc, wcap, mode);
    std::vector<float> qv(q, q + dim);
    int *result; float *dist; int sum, e = 0;
    if (mode == 2 || mode == 3) {
        OSC &m = mode == 2 ? m2 : static_cast<OSC &>(m3);
        m.set_index(dim, mc, kc, mp, kp, N, cq, pq, L, pid, codes, raw);
        m.pre_compute1();
        sum = run_one(m, nullptr, &m, mode, s, qv.data(), R, w, T, kc, real_dist != 0, result,
                      dist, &e);
        m.release(true);
    } else {
        m1.set_index(dim, mc, kc, mp, kp, N, cq, pq, L, pid, codes, raw);
        m1.pre_compute1();
        sum = run_one(m1, &m1, nullptr, mode, s, qv.data(), R, w, T, kc, real_dist != 0, result,
                      dist, &e);
        m1.release(true);
    }
    if (empty_out) *empty_out = e;
    if (sum > cap) sum = -1;
    else if (sum > 0) {
        memcpy(ids_all, result, sizeof(int) * (size_t)sum);
        memcpy(dist_all, dist, sizeof(float) * (size_t)sum);
    }
    ::operator delete(result);
    ::operator delete(dist);
    return sum;
}

/* pre_compute1 then pre_compute2(q) of the reference; copies the five tables. */
int ref_tables(int dim, int mc, int kc, int mp, int kp,
               float *cq, float *pq, const float *q,
               float *norm_c, float *norm_r, float *dot_cr, float *diff_qc, float *diff_qr) {
    OMulti m;
    m.set_index(dim, mc, kc, mp, kp, 0, cq, pq, nullptr, nullptr, nullptr, nullptr);
    m.pre_compute1();
    std::vector<float> qv(q, q + dim);
    m.pre_compute2(qv.data());
    memcpy(norm_c, m.get_norm_c(), sizeof(float) * (size_t)mc * kc);
    memcpy(norm_r, m.get_norm_r(), sizeof(float) * (size_t)mp * kp);
    memcpy(dot_cr, m.get_dot_cr(), sizeof(float) * (size_t)kc * kp * mp);
    memcpy(diff_qc, m.get_diff_qc(), sizeof(float) * (size_t)mc * kc);
    memcpy(diff_qr, m.get_diff_qr(), sizeof(float) * (size_t)mp * kp);
    m.release(true);
    return 0;
}

/* Encoder::encode<float> / SCEncoder::encode<float> on an .fvecs file with
 * the codebooks of two .ctr_ files; copies cid and codes.  nc = 0 selects the
 * IVF/IMI encoder, nc >= 2 the SC encoder with nc nearest centroids. */
struct OEnc : public Encoder {
    unsigned short *get_cid() { return cid; }
    unsigned char *get_codes() { return codes; }
    int get_N() { return config.N; }
    int get_mc() { return config.mc; }
    int get_mp() { return config.mp; }
};
struct OSCEnc : public SCEncoder {
    explicit OSCEnc(int nc) : SCEncoder(nc) {}
    unsigned short *get_cid() { return cid; }
    unsigned char *get_codes() { return codes; }
    int get_N() { return config.N; }
    int get_mp() { return config.mp; }
};

int ref_encode(const char *cq_path, const char *pq_path, const char *fvecs_path, int nc,
               int nthreads, unsigned short *cid_out, unsigned char *codes_out, long cap_rows) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    if (nc == 0) {
        OEnc e;
        e.load_codebooks(cq_path, pq_path, false);
        e.encode<float>(fvecs_path, 4, false);
        long n = e.get_N();
        if (n > cap_rows) return -1;
        memcpy(cid_out, e.get_cid(), sizeof(unsigned short) * (size_t)n * e.get_mc());
        memcpy(codes_out, e.get_codes(), (size_t)n * e.get_mp());
        return (int)n;
    }
    OSCEnc e(nc);
    e.load_codebooks(cq_path, pq_path, false);
    e.encode<float>(fvecs_path, 4, false);
    long n = e.get_N();
    if (n > cap_rows) return -1;
    memcpy(cid_out, e.get_cid(), sizeof(unsigned short) * (size_t)n * nc);
    memcpy(codes_out, e.get_codes(), (size_t)n * e.get_mp());
    return (int)n;
}

/* Encoder (nc = 0) or SCEncoder (nc = 2) encode + distribution + output:
 * writes the reference's own .edat_ file into db_path with prefix. */
int ref_build_edat(const char *cq_path, const char *pq_path, const char *fvecs_path, int nc,
                   const char *db_path, const char *prefix) {
    if (nc == 0) {
        OEnc e;
        e.load_codebooks(cq_path, pq_path, false);
        e.encode<float>(fvecs_path, 4, false);
        e.distribution(false);
        e.output(db_path, prefix, false);
        return 0;
    }
    OSCEnc e(nc);
    e.load_codebooks(cq_path, pq_path, false);
    e.encode<float>(fvecs_path, 4, false);
    e.distribution(false);
    e.output(db_path, prefix, false);
    return 0;
}

/* Evaluation::calc_recall (evaluation.h:58-92) and calc_comb_recall
 * (evaluation.h:103-140) of the reference, on caller arrays. */
int ref_calc_recall(int *result, int *gt, int R, int N) {
    Evaluation e;
    int recall = 0;
    e.calc_recall(result, gt, R, N, recall, false);
    return recall;
}

int ref_calc_comb_recall(int **results, int *gt, int R, int N, int S) {
    Evaluation e;
    int recall = 0;
    e.calc_comb_recall(results, gt, R, N, S, recall, false);
    return recall;
}

} // extern "C"
