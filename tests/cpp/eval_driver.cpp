// Drives the drop-in Evaluation (second-candidate_b200/cpp/evaluation.h) the
// way the reference's test_evaluation.cpp drives its own: reads N R S, then S
// result arrays of N*R ids and N ground-truth ids (text, stdin), prints the
// calc_recall count of the first array and the calc_comb_recall count of all.
#include <iostream>
#include <vector>

#include "evaluation.h"

int main() {
    int N = 0, R = 0, S = 0;
    std::cin >> N >> R >> S;
    std::vector<std::vector<int>> res((size_t)S, std::vector<int>((size_t)N * R));
    for (auto &r : res)
        for (auto &x : r) std::cin >> x;
    std::vector<int> gt((size_t)N);
    for (auto &x : gt) std::cin >> x;
    std::vector<int *> ptrs;
    for (auto &r : res) ptrs.push_back(r.data());
    SC::Evaluation e;
    int recall = 0, comb = 0;
    e.calc_recall(ptrs[0], gt.data(), R, N, recall, false);
    e.calc_comb_recall(ptrs.data(), gt.data(), R, N, S, comb, false);
    std::cout << recall << " " << comb << std::endl;
    return 0;
}
