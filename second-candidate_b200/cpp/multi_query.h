/*
 * multi_query.h -- drop-in for the reference's MultiQuery
 * (include/multi_query.h:36-53): search_multi2 with the same argument list.
 * The scratch arrays are accepted and left untouched (the device keeps its
 * own per-query state), so `traversed` stays clean as the reference leaves
 * it; `e` receives the number of empty cells visited and t1/t2 accumulate the
 * device time of the table build and of the selection + scan (clock ticks).
 */
#ifndef SCG_DROPIN_MULTI_QUERY_H_
#define SCG_DROPIN_MULTI_QUERY_H_

#include "query.h"

namespace SC {

class MultiQuery : public PQQuery {
public:
    MultiQuery() : PQQuery() {}
    virtual ~MultiQuery() {}

    /* MultiQuery::search_multi2 (multi_query.h:62-273).  M < kc confines the
     * walk to ranks 0..M-1 of both coarse lists (the reference sorts only
     * those, multi_query.h:125-128); where its walk stays inside them the
     * results agree. */
    void search_multi2(float *query, float *&v_tmp, float *&dist, float *&q, int *tmp, int *&result, int *&hid1,
                       int *&hid2, int *&hid3, int *&hid4, int *&s1, int *&s2, int *&prebuck, int *&cache,
                       bool *traversed, int &sum, int R, int w, int T, int M, int &e, double &t1, double &t2,
                       bool real_dist, bool verbose) {
        (void)v_tmp; (void)q; (void)tmp; (void)hid1; (void)hid2; (void)hid3; (void)hid4; (void)s1; (void)s2;
        (void)prebuck; (void)cache; (void)traversed; (void)verbose;
        if (config.mc != 2) {
            std::cerr << "This search method is for Multi-D-ADC-2 only" << std::endl;
            return;
        }
        run_one(SCG_IMI, query, R, w, T, real_dist, dist, result, sum, &e, &t1, &t2, M);
    }
};

}  // namespace SC
#endif
