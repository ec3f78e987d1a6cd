/*
 * query.h -- drop-in for the reference's PQQuery (include/query.h:45-80) over
 * the B200 library (scg.h).  Same class name, methods and argument meaning;
 * the index lives on the GPU and each search call runs the batched device
 * search for one query.
 *
 * Differences a caller can see:
 *  - pre_compute2 is a no-op: the per-query tables are built on the device
 *    inside each search (with the reference's float order);
 *  - result/dist are still allocated by the callee with ::operator new
 *    (sized `sum`, freed by the caller with ::delete), but only their first
 *    min(R, sum) entries are filled -- the R best in ascending distance,
 *    equal distances by id; the rest hold -1 / +inf.  The reference fills
 *    all `sum` entries but documents only the first min(R, sum);
 *  - R is limited to 1024.
 * Wrong-mode calls print the reference's message to cerr and return with the
 * outputs untouched; I/O failures end the process like the reference.
 */
#ifndef SCG_DROPIN_QUERY_H_
#define SCG_DROPIN_QUERY_H_

#include <cmath>
#include <ctime>
#include <limits>

#include "sc_algorithm.h"
#include "sc_utilities.h"

namespace SC {

class PQQuery {
protected:
    scg_index *h = nullptr;
    int size = 0;
    int not_empty = 0;
    PQConfig config;
    int nc_ = 0;             // cells are kc^nc_ (second-candidate: 2)
    int precision_ = SCG_FP32_EXACT;
    float *raw_data = nullptr;

    /* One query through the device search; fills the reference-style
     * outputs.  M > 0: the walk uses only ranks 0..M-1 of each sorted
     * coarse list.  Returns false (after printing) on a library error. */
    bool run_one(int mode, float *query, int R, int w, int T, bool real_dist, float *&dist, int *&result,
                 int &sum, int *empty = nullptr, double *t_tables = nullptr, double *t_search = nullptr,
                 int M = 0) {
        if (scg_set_rank_limit(h, M) != SCG_OK) {
            std::cerr << scg_message() << std::endl;
            return false;
        }
        scg_search_params p;
        p.mode = mode;
        p.R = R;
        p.w = w;
        p.T = T;
        p.precision = precision_;
        p.rerank = real_dist ? -1 : 0;
        std::vector<int> ids((size_t)R);
        std::vector<float> d((size_t)R);
        int s = 0;
        if (scg_search(h, &p, query, 1, ids.data(), d.data(), &s) != SCG_OK) {
            std::cerr << scg_message() << std::endl;
            return false;
        }
        sum = s;
        if (s > 0) {
            result = (int *)::operator new(sizeof(int) * (size_t)s);
            dist = (float *)::operator new(sizeof(float) * (size_t)s);
            int m = s < R ? s : R;
            for (int i = 0; i < s; i++) {
                result[i] = i < m ? ids[(size_t)i] : -1;
                dist[i] = i < m ? d[(size_t)i] : std::numeric_limits<float>::infinity();
            }
        }
        if (empty) scg_last_query_stats(h, nullptr, empty, 1);
        if (t_tables || t_search) {
            float ms[2] = {0, 0};
            scg_last_timings(h, ms, 2);
            if (t_tables) *t_tables += ms[0] * 1e-3 * CLOCKS_PER_SEC;
            if (t_search) *t_search += ms[1] * 1e-3 * CLOCKS_PER_SEC;
        }
        return true;
    }

public:
    PQQuery() {
        memset(&config, 0, sizeof(config));
        if (scg_index_create(&h, 0) != SCG_OK) scg_die("cannot create the GPU index");
    }
    virtual ~PQQuery() {
        scg_index_destroy(h);
        ::operator delete(raw_data);
    }

    /* PQQuery::load_codebooks (query.cpp:66-75). */
    void load_codebooks(const char *cq_path, const char *pq_path, bool verbose) {
        if (scg_load_codebooks_file(h, cq_path, pq_path) != SCG_OK) scg_die("Cannot load the codebooks");
        int64_t n = 0;
        scg_index_info(h, &config.dim, &config.mc, &config.kc, &config.mp, &config.kp, &n);
        size = (int)std::pow((double)config.kc, (double)config.mc);
        std::cout << "--> Settings: (kc,mc,kp,mp)=" << config.kc << " " << config.mc << " " << config.kp << " "
                  << config.mp << std::endl;
        (void)verbose;
    }

    /* PQQuery::load_encoded_data (query.cpp:82-165). */
    int load_encoded_data(const char *filename, bool verbose) {
        int nc = nc_ ? nc_ : config.mc;
        if (scg_load_encoded_file(h, filename, nc) != SCG_OK) scg_die("Cannot load the encoded data");
        int64_t n = 0;
        scg_index_info(h, nullptr, nullptr, nullptr, nullptr, nullptr, &n);
        config.N = (int)n;
        int64_t cells = 1;
        for (int i = 0; i < nc; i++) cells *= config.kc;
        std::vector<int> L((size_t)cells);
        scg_cell_counts(h, L.data(), cells);
        not_empty = 0;
        for (int64_t c = 0; c < cells; c++) not_empty += (L[(size_t)c] - (c ? L[(size_t)c - 1] : 0)) > 0;
        cached_L_.swap(L);
        if (verbose) std::cout << "The number of non empty buckets: " << not_empty << std::endl;
        return config.N;
    }

    /* PQQuery::load_data (query.h:82-86): raw vectors for the exact branch. */
    template <typename DataType>
    void load_data(const char *filename, int offset, bool verbose) {
        ::operator delete(raw_data);
        raw_data = nullptr;
        config.N = load_and_convert_data<DataType, float>(filename, raw_data, offset, config.dim, verbose);
        if (scg_load_raw(h, raw_data, config.N) != SCG_OK) std::cerr << scg_message() << std::endl;
    }

    /* PQQuery::pre_compute1 (query.h:91-149). */
    void pre_compute1() {
        if (scg_precompute(h) != SCG_OK) scg_die("pre_compute1");
    }
    /* PQQuery::pre_compute2 (query.h:154-184): built on the device per search. */
    void pre_compute2(float *) {}

    /* PQQuery::search_ivfadc (query.h:202-325). */
    void search_ivfadc(float *query, float *&v_tmp, float *&dist, int *&result, int *&buckets, int *&prebuck,
                       int &sum, int R, int w, int T, bool real_dist, bool verbose) {
        (void)v_tmp; (void)buckets; (void)prebuck; (void)verbose;
        if (config.mc != 1) {
            std::cerr << "This search method is for IVFADC only" << std::endl;
            return;
        }
        run_one(SCG_IVFADC, query, R, w, T, real_dist, dist, result, sum);
    }

    int get_size() { return not_empty; }
    int get_full_size() { return size; }

    /* PQQuery::entropy (query.cpp:168-182). */
    double entropy(size_t n) {
        double e = 0.0, N = config.N;
        for (size_t i = 0; i < n && i < cached_L_.size(); i++) {
            double l = cached_L_[i] - (i ? cached_L_[i - 1] : 0);
            if (l > 0) {
                double x = N / l;
                e += std::log2(x) / x;
            }
        }
        return e;
    }

    /* Additions of the B200 build: the batched entry point and the handle. */
    int search_batch(int mode, const float *Q, int nq, int R, int w, int T, int *ids, float *dists, int *sums,
                     int M = 0) {
        int rc = scg_set_rank_limit(h, M);
        if (rc != SCG_OK) return rc;
        scg_search_params p;
        p.mode = mode; p.R = R; p.w = w; p.T = T; p.precision = precision_; p.rerank = 0;
        return scg_search(h, &p, Q, nq, ids, dists, sums);
    }
    void set_precision(int p) { precision_ = p; }
    scg_index *handle() { return h; }

protected:
    std::vector<int> cached_L_;
};

}  // namespace SC
#endif
