/*
 * quantizer.h -- drop-in for the reference's PQQuantizer<DataType>
 * (include/quantizer.h:47-106): the same members and methods.
 * create_sub_quantizers clusters the `part` strips of the data on the GPU
 * (scg_kmeans: k-means++ seeding and Lloyd steps with FP64 means, all strips
 * at once) instead of greg_kmeans, whose Lloyd loop stops after one pass;
 * output writes the same .ctr_ file (quantizer.h:357-431: float {nsc, part,
 * dim} then the centres); calc_residual_vector subtracts, per loaded coarse
 * codebook and part, the first nearest centroid under float-rounded
 * distance_l2_square comparisons (quantizer.h:456-510).
 */
#ifndef SCG_DROPIN_QUANTIZER_H_
#define SCG_DROPIN_QUANTIZER_H_

#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>

#include "sc_utilities.h"

namespace SC {

template <typename DataType>
class PQQuantizer {
protected:
    int dim, part, nsc, offset;
    int N;
    float *centers;  // [part][nsc][dim / part]
    int *labels;     // [part][N]
    float **cq;      // loaded coarse codebooks (load_codebooks)
    int k;
    int *kc, *mc;

public:
    float *data;  // [N][dim]
    int iterations = 25;       // Lloyd steps after the k-means++ seeding
    unsigned long long seed = 1234;
    int device = 0;

    PQQuantizer(int _dim, int _m, int _nsc, int _os, bool verbose)
        : dim(_dim), part(_m), nsc(_nsc), offset(_os), N(0), centers(nullptr), labels(nullptr), cq(nullptr), k(0),
          kc(nullptr), mc(nullptr), data(nullptr) {
        if (dim <= 0 || part <= 0 || dim % part != 0) {
            if (verbose) std::cerr << "Error at parameters of PQQuantizer" << std::endl;
            exit(EXIT_FAILURE);
        }
        centers = (float *)::operator new(sizeof(float) * (size_t)nsc * dim);
    }

    PQQuantizer(int _dim, int _m, int _nsc, int _os, int _k, bool verbose) : PQQuantizer(_dim, _m, _nsc, _os, verbose) {
        k = _k;
        cq = (float **)::operator new(sizeof(float *) * (size_t)(k > 0 ? k : 1));
        for (int i = 0; i < k; i++) cq[i] = nullptr;
        kc = (int *)::operator new(sizeof(int) * (size_t)(k > 0 ? k : 1));
        mc = (int *)::operator new(sizeof(int) * (size_t)(k > 0 ? k : 1));
    }

    virtual ~PQQuantizer() {
        ::operator delete(centers);
        ::operator delete(labels);
        ::operator delete(data);
        for (int i = 0; i < k; i++) ::operator delete(cq[i]);
        ::operator delete(cq);
        ::operator delete(kc);
        ::operator delete(mc);
    }

    void load_data(const char *filename, bool verbose) {
        N = load_and_convert_data<DataType, float>(filename, data, offset, dim, verbose);
        ::operator delete(labels);
        labels = (int *)::operator new(sizeof(int) * (size_t)N * part);
        if (verbose) std::cout << "Initialized " << N << " vectors" << std::endl;
    }

    void load_data_mat(float *_data, int _N) {
        if (_N > 0) N = _N;
        data = _data;
        ::operator delete(labels);
        labels = (int *)::operator new(sizeof(int) * (size_t)N * part);
    }

    void create_sub_quantizers(bool verbose) {
        int rc = scg_kmeans(data, N, dim, part, nsc, iterations, seed, centers, labels, device);
        if (rc) {
            if (verbose) std::cerr << "k-means failed: " << scg_message() << std::endl;
            exit(EXIT_FAILURE);
        }
        if (verbose) std::cout << "Finished " << part << " sub-codebooks" << std::endl;
    }

    // sqrt of the sum over strips of (sqrt of the strip's summed squared
    // distances)^2 (quantizer.h:277-300 with SimpleCluster::distortion).
    double distortion(bool) {
        const int bs = dim / part;
        double e = 0.0;
        for (int i = 0; i < part; i++) {
            float es = 0.0f;
            const float *c = centers + (size_t)i * nsc * bs;
            for (int j = 0; j < N; j++) {
                const float *x = data + (size_t)j * dim + (size_t)i * bs;
                const float *cc = c + (size_t)labels[(size_t)i * N + j] * bs;
                double d = 0.0;
                for (int t = 0; t < bs; t++) {
                    const double tmp = (double)(x[t] - cc[t]);
                    d += tmp * tmp;
                }
                es += (float)d;
            }
            const double s = std::sqrt((double)es);
            e += s * s;
        }
        return std::sqrt(e);
    }

    int size() { return N; }

    float *get_center_at(int id, bool) { return centers + (size_t)id * nsc * (dim / part); }
    int *get_label_at(int id, bool) { return labels + (size_t)id * N; }

    void set_params(int _k, int _m, int _nsc) {
        for (int i = 0; i < k; i++) ::operator delete(cq[i]);
        ::operator delete(cq);
        ::operator delete(kc);
        ::operator delete(mc);
        k = _k;
        cq = (float **)::operator new(sizeof(float *) * (size_t)(k > 0 ? k : 1));
        for (int i = 0; i < k; i++) cq[i] = nullptr;
        kc = (int *)::operator new(sizeof(int) * (size_t)(k > 0 ? k : 1));
        mc = (int *)::operator new(sizeof(int) * (size_t)(k > 0 ? k : 1));
        part = _m;
        nsc = _nsc;
        if (dim <= 0 || part <= 0 || dim % part != 0) {
            std::cerr << "Error at parameters of PQQuantizer" << std::endl;
            exit(EXIT_FAILURE);
        }
        ::operator delete(centers);
        centers = (float *)::operator new(sizeof(float) * (size_t)nsc * dim);
        ::operator delete(labels);
        labels = (int *)::operator new(sizeof(int) * (size_t)(N > 0 ? N : 1) * part);
    }

    // filename.ctr_: float {nsc, part, dim}, then nsc * dim floats.
    void output(const char *filename, bool) {
        char fn[1024];
        snprintf(fn, sizeof(fn), "%s.ctr_", filename);
        FILE *f = fopen(fn, "wb");
        if (!f) {
            std::cerr << "Cannot open the file " << fn << std::endl;
            exit(EXIT_FAILURE);
        }
        const float hdr[3] = {(float)nsc, (float)part, (float)dim};
        fwrite(hdr, sizeof(float), 3, f);
        fwrite(centers, sizeof(float), (size_t)nsc * dim, f);
        fclose(f);
    }

    void load_codebooks(char **filename, bool verbose) {
        for (int i = 0; i < k; i++) {
            PQConfig config;
            ::operator delete(cq[i]);
            cq[i] = nullptr;
            load_codebook<float>(filename[i], config, cq[i], 0, verbose);
            kc[i] = config.kc;
            mc[i] = config.mc;
        }
    }

    // data -= the nearest centroid of each part of each loaded codebook.
    void calc_residual_vector(bool) {
        for (int k0 = 0; k0 < k; k0++) {
            const int m = mc[k0], bs = dim / m, kk = kc[k0];
            for (int i = 0; i < N; i++) {
                float *x = data + (size_t)i * dim;
                const float *c = cq[k0];
                for (int j = 0; j < m; j++) {
                    float d = FLT_MAX;
                    int pos = 0;
                    for (int k1 = 0; k1 < kk; k1++) {
                        const float dt = (float)distance_l2_square(x, c + (size_t)k1 * bs, bs);
                        if (d > dt) {
                            d = dt;
                            pos = k1;
                        }
                    }
                    const float *cc = c + (size_t)pos * bs;
                    for (int t = 0; t < bs; t++) x[t] -= cc[t];
                    c += (size_t)kk * bs;
                    x += bs;
                }
            }
        }
    }
};

}  // namespace SC

#endif
