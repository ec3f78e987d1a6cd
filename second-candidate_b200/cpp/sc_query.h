/*
 * sc_query.h -- drop-in for the reference's SCQuery (include/sc_query.h:21-51):
 * the second-candidate search over ordered pairs of nearest coarse centroids.
 * search_mr_ivf and search_mr_ivf3 return their R best in ascending distance
 * (the reference leaves them unsorted, sc_query.h:250-252, :469-473).
 */
#ifndef SCG_DROPIN_SC_QUERY_H_
#define SCG_DROPIN_SC_QUERY_H_

#include "query.h"

namespace SC {

class SCQuery : public PQQuery {
protected:
    int nc;

public:
    SCQuery() : PQQuery(), nc(2) { nc_ = 2; }
    explicit SCQuery(int n) : PQQuery(), nc(n) { nc_ = n; }
    virtual ~SCQuery() {}

    /* SCQuery::load_encoded_data (sc_query.cpp:36-123): kc^nc cells. */
    int load_encoded_data(const char *filename, bool verbose) { return PQQuery::load_encoded_data(filename, verbose); }

    /* SCQuery::search_mr_ivf (sc_query.h:60-256).  M < kc confines the walk
     * to ranks 0..M-1 of the sorted coarse list (sc_query.h:105-106 sorts
     * only those). */
    void search_mr_ivf(float *query, float *&v_tmp, float *&dist, int *tmp, int *&result, int *&hid1, int *&hid2,
                       int *&hid3, int *&hid4, int *&s1, int *&s2, int *&prebuck, int *&cache, bool *traversed,
                       int &sum, int R, int w, int T, int M, bool real_dist, bool verbose) {
        (void)v_tmp; (void)tmp; (void)hid1; (void)hid2; (void)hid3; (void)hid4; (void)s1; (void)s2; (void)prebuck;
        (void)cache; (void)traversed; (void)verbose;
        if (config.mc != 1 || nc != 2) {
            std::cerr << "This search method is for MultiRank IVFADC only" << std::endl;
            return;
        }
        run_one(SCG_SC2, query, R, w, T, real_dist, dist, result, sum, nullptr, nullptr, nullptr, M);
    }

    /* SCQuery::search_mr_ivf3 (sc_query.h:265-475): the three-nearest-centroid
     * cells of an SCQuery(3) index, walked over rank triples (ranks 0..M-1
     * for M < kc). */
    void search_mr_ivf3(float *query, float *&v_tmp, float *&dist, int *tmp, int *&result, int *&hid1, int *&hid2,
                        int *&hid3, int *&hid4, int *&hid5, int *&hid6, int *&s1, int *&prebuck, int *&cache,
                        bool *traversed, int &sum, int R, int w, int T, int M, bool real_dist, bool verbose) {
        (void)v_tmp; (void)tmp; (void)hid1; (void)hid2; (void)hid3; (void)hid4; (void)hid5; (void)hid6; (void)s1;
        (void)prebuck; (void)cache; (void)traversed; (void)verbose;
        if (config.mc != 1 || nc != 3) {
            std::cerr << "This search method is for MultiRank IVFADC-3 only" << std::endl;
            return;
        }
        run_one(SCG_SC3, query, R, w, T, real_dist, dist, result, sum, nullptr, nullptr, nullptr, M);
    }
};

}  // namespace SC
#endif
