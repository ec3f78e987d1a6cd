/*
 * evaluation.h -- drop-in for the reference's Evaluation
 * (include/evaluation.h:20-25): ground truth (first column of an .ivecs
 * file) and recall@R = the number of queries whose true nearest neighbour is
 * among their first R results (evaluation.h:58-92).
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
};
}  // namespace SC
#endif
