/*
 * evaluation.h -- drop-in for the reference's Evaluation
 * (include/evaluation.h:20-25): ground truth (first column of an .ivecs
 * file), recall@R = the number of queries whose true nearest neighbour is
 * among their first R results (evaluation.h:58-92), and the same over the
 * union of several result sets (evaluation.h:103-140).
 */
#ifndef SCG_DROPIN_EVALUATION_H_
#define SCG_DROPIN_EVALUATION_H_

#include "sc_utilities.h"

namespace SC {
class Evaluation {
public:
    void load_groundtruth(const char *filename, int *&gt, int d, int &N, bool verbose) {
        int *tmp = nullptr;
        N = load_data<int>(filename, tmp, 4, d, verbose);
        gt = (int *)::operator new(sizeof(int) * (size_t)(N > 0 ? N : 1));
        for (int i = 0; i < N; i++) gt[i] = tmp[(size_t)i * d];
        ::operator delete(tmp);
    }
    void calc_recall(int *result, int *groundtruth, int R, int N, int &recall, bool verbose) {
        recall = 0;
        for (int i = 0; i < N; i++) {
            for (int j = 0; j < R; j++)
                if (result[(size_t)i * R + j] == groundtruth[i]) {
                    recall++;
                    break;
                }
        }
        if (verbose) std::cout << "Recall@" << R << " = " << recall << std::endl;
    }
    /* Evaluation::calc_comb_recall (evaluation.h:103-140): the number of
     * queries whose true nearest neighbour is among the first R results of
     * any of the S result arrays results[0..S) (each [N][R]). */
    void calc_comb_recall(int **results, int *groundtruth, int R, int N, int S, int &recall, bool verbose) {
        recall = 0;
        for (int i = 0; i < N; i++) {
            bool found = false;
            for (int j = 0; j < S && !found; j++)
                for (int k = 0; k < R; k++)
                    if (results[j][(size_t)i * R + k] == groundtruth[i]) {
                        found = true;
                        break;
                    }
            if (found) recall++;
        }
        if (verbose) std::cout << "Recall@" << R << " = " << recall << std::endl;
    }
};
}  // namespace SC
#endif
