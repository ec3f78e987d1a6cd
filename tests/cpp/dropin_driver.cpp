// Drives the drop-in headers the way the reference's own test drivers drive
// the reference classes (test_query.cpp:147-196, test_multi_query.cpp:146-213,
// test_sc_query.cpp:111-203, test_encoder.cpp:58-88): one query per call with
// caller-owned scratch, results freed with ::delete.
//
//   dropin_driver search <ivf|imi|sc|sc3> <cq.ctr_> <pq.ctr_> <x.edat_> <q.fvecs> <dim> <R> <w> <T> <out.txt>
//                        [<base.fvecs>|- [M]]   (base: load_data + real_dist = true; M: the coarse-list argument)
//   dropin_driver encode <0|2> <cq.ctr_> <pq.ctr_> <x.fvecs> <outdir> <prefix>
//   dropin_driver quantize <x.fvecs> <dim> <m> <nsc> <out_prefix>      (PQQuantizer, test_quantizer.cpp-style)
//   dropin_driver residual <pq|sc> <x.fvecs> <dim> <m> <cq.ctr_> <out.fvecs>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>

#include "evaluation.h"
#include "multi_query.h"
#include "sc_encoder.h"
#include "sc_quantizer.h"
#include "sc_query.h"

using namespace SC;

static int search(int argc, char **argv) {
    const char *mode = argv[2];
    int d = atoi(argv[7]), R = atoi(argv[8]), w = atoi(argv[9]), T = atoi(argv[10]);
    const char *base = argc > 12 && strcmp(argv[12], "-") ? argv[12] : nullptr;
    const bool real_dist = base != nullptr;
    const int M_arg = argc > 13 ? atoi(argv[13]) : 0;
    float *data = nullptr;
    int N = load_and_convert_data<float, float>(argv[6], data, 4, d, false);
    std::ofstream out(argv[11]);
    out << std::setprecision(9);
    int sum = 0, bad = 0;
    int *result = nullptr;
    float *dist = nullptr;
    if (!strcmp(mode, "imi")) {
        MultiQuery q;
        q.load_codebooks(argv[3], argv[4], false);
        q.load_encoded_data(argv[5], false);
        if (base) q.load_data<float>(base, 4, false);
        q.pre_compute1();
        int kc = q.get_full_size() > 0 ? (int)(0.5 + std::sqrt((double)q.get_full_size())) : 0;
        const int M = M_arg > 0 ? M_arg : kc;
        float *v_tmp = new float[2 * kc + w], *q2 = new float[2];
        int *it = new int[2 * kc], *h1 = new int[w], *h2 = new int[w], *h3 = new int[w], *h4 = new int[w];
        int *s1 = new int[w], *s2 = new int[w], *pb = new int[w], *cache = new int[w];
        bool *trav = new bool[(size_t)kc * kc]();
        double t1 = 0, t2 = 0;
        for (int i = 0; i < N; i++) {
            int e = 0;
            q.search_multi2(data + (size_t)i * d, v_tmp, dist, q2, it, result, h1, h2, h3, h4, s1, s2, pb, cache,
                            trav, sum, R, w, T, M, e, t1, t2, real_dist, false);
            if (trav[0]) bad++;  // test_multi_query.cpp:191
            out << sum << " " << e;
            for (int j = 0; j < (R > sum ? sum : R); j++) out << " " << result[j] << ":" << dist[j];
            out << "\n";
            ::operator delete(result);
            ::operator delete(dist);
            result = nullptr;
            dist = nullptr;
        }
    } else if (!strcmp(mode, "sc3")) {
        SCQuery q(3);
        q.load_codebooks(argv[3], argv[4], false);
        q.load_encoded_data(argv[5], false);
        if (base) q.load_data<float>(base, 4, false);
        q.pre_compute1();
        int kc = q.get_full_size();
        const int M = M_arg > 0 ? M_arg : kc;
        float *v_tmp = new float[kc + w];
        int *it = new int[kc], *h1 = new int[w], *h2 = new int[w], *h3 = new int[w], *h4 = new int[w];
        int *h5 = new int[w], *h6 = new int[w], *s1 = new int[w], *pb = new int[w];
        int *cache = new int[(size_t)kc * kc * kc + w];
        bool *trav = new bool[(size_t)kc * kc * kc]();
        for (int i = 0; i < N; i++) {
            q.search_mr_ivf3(data + (size_t)i * d, v_tmp, dist, it, result, h1, h2, h3, h4, h5, h6, s1, pb, cache,
                             trav, sum, R, w, T, M, real_dist, false);
            out << sum << " 0";
            for (int j = 0; j < (R > sum ? sum : R); j++) out << " " << result[j] << ":" << dist[j];
            out << "\n";
            ::operator delete(result);
            ::operator delete(dist);
            result = nullptr;
            dist = nullptr;
        }
    } else if (!strcmp(mode, "sc")) {
        SCQuery q;
        q.load_codebooks(argv[3], argv[4], false);
        q.load_encoded_data(argv[5], false);
        if (base) q.load_data<float>(base, 4, false);
        q.pre_compute1();
        int kc = q.get_full_size();
        const int M = M_arg > 0 ? M_arg : kc;
        float *v_tmp = new float[kc + w];
        int *it = new int[kc], *h1 = new int[w], *h2 = new int[w], *h3 = new int[w], *h4 = new int[w];
        int *s1 = new int[w], *s2 = new int[w], *pb = new int[w], *cache = new int[w];
        bool *trav = new bool[(size_t)kc * kc]();
        trav[0] = true;  // test_sc_query.cpp:160-161
        for (int i = 0; i < N; i++) {
            q.search_mr_ivf(data + (size_t)i * d, v_tmp, dist, it, result, h1, h2, h3, h4, s1, s2, pb, cache, trav,
                            sum, R, w, T, M, real_dist, false);
            if (!trav[0] || trav[1]) bad++;  // test_sc_query.cpp:182-183
            out << sum << " 0";
            for (int j = 0; j < (R > sum ? sum : R); j++) out << " " << result[j] << ":" << dist[j];
            out << "\n";
            ::operator delete(result);
            ::operator delete(dist);
            result = nullptr;
            dist = nullptr;
        }
    } else {
        PQQuery q;
        q.load_codebooks(argv[3], argv[4], false);
        q.load_encoded_data(argv[5], false);
        if (base) q.load_data<float>(base, 4, false);
        q.pre_compute1();
        int kc = q.get_full_size();
        float *v_tmp = new float[kc];
        int *buckets = new int[kc], *bk = new int[kc];
        for (int i = 0; i < N; i++) {
            q.search_ivfadc(data + (size_t)i * d, v_tmp, dist, result, buckets, bk, sum, R, w, T, real_dist, false);
            out << sum << " 0";
            for (int j = 0; j < (R > sum ? sum : R); j++) out << " " << result[j] << ":" << dist[j];
            out << "\n";
            ::operator delete(result);
            ::operator delete(dist);
            result = nullptr;
            dist = nullptr;
        }
    }
    ::operator delete(data);
    if (bad) {
        std::cerr << "traversed invariant broken " << bad << " times" << std::endl;
        return 2;
    }
    return 0;
}

static int encode(int argc, char **argv) {
    int nc = atoi(argv[2]);
    if (nc == 0) {
        Encoder e;
        e.load_codebooks(argv[3], argv[4], false);
        e.encode<float>(argv[5], 4, false);
        e.distribution(false);
        e.output(argv[6], argv[7], false);
    } else {
        SCEncoder e(nc);
        e.load_codebooks(argv[3], argv[4], false);
        e.encode<float>(argv[5], 4, false);
        e.distribution(false);
        e.output(argv[6], argv[7], false);
    }
    return 0;
}

// Trains `m` sub-codebooks of `nsc` centres on the rows of x.fvecs, writes
// out_prefix.ctr_ and prints the distortion.
static int quantize(int, char **argv) {
    const int dim = atoi(argv[3]), m = atoi(argv[4]), nsc = atoi(argv[5]);
    PQQuantizer<float> q(dim, m, nsc, 4, false);
    q.load_data(argv[2], false);
    q.create_sub_quantizers(false);
    q.output(argv[6], false);
    std::cout << std::setprecision(17) << q.distortion(false) << std::endl;
    return 0;
}

// Subtracts the nearest (pq) or second-nearest (sc) centroid of the coarse
// codebook cq.ctr_ from every part of every row; writes the rows as fvecs.
static int residual(int, char **argv) {
    const bool sc = !strcmp(argv[2], "sc");
    const int dim = atoi(argv[4]), m = atoi(argv[5]);
    char *files[1] = {argv[6]};
    PQQuantizer<float> *q = sc ? new SCQuantizer<float>(dim, m, 1, 4, 1, false) : new PQQuantizer<float>(dim, m, 1, 4, 1, false);
    q->load_data(argv[3], false);
    q->load_codebooks(files, false);
    if (sc) static_cast<SCQuantizer<float> *>(q)->calc_residual_vector(false);
    else q->calc_residual_vector(false);
    FILE *f = fopen(argv[7], "wb");
    for (int i = 0; i < q->size(); i++) {
        fwrite(&dim, sizeof(int), 1, f);
        fwrite(q->data + (size_t)i * dim, sizeof(float), (size_t)dim, f);
    }
    fclose(f);
    delete q;
    return 0;
}

int main(int argc, char **argv) {
    if (argc >= 12 && !strcmp(argv[1], "search")) return search(argc, argv);
    if (argc >= 8 && !strcmp(argv[1], "encode")) return encode(argc, argv);
    if (argc >= 7 && !strcmp(argv[1], "quantize")) return quantize(argc, argv);
    if (argc >= 8 && !strcmp(argv[1], "residual")) return residual(argc, argv);
    std::cerr << "usage: see the header of dropin_driver.cpp" << std::endl;
    return 1;
}
