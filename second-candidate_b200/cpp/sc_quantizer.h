/*
 * sc_quantizer.h -- drop-in for the reference's SCQuantizer<DataType>
 * (include/sc_quantizer.h:28-37): a PQQuantizer whose residual, per part,
 * subtracts the SECOND nearest centroid of each loaded coarse codebook
 * (sc_quantizer.h:72-132, float-rounded distance_l2_square comparisons, the
 * runner-up tracked as in the reference's update order).
 */
#ifndef SCG_DROPIN_SC_QUANTIZER_H_
#define SCG_DROPIN_SC_QUANTIZER_H_

#include "quantizer.h"

namespace SC {

template <typename DataType>
class SCQuantizer : public PQQuantizer<DataType> {
public:
    SCQuantizer(int _dim, int _m, int _nsc, int _os, int _k, bool verbose)
        : PQQuantizer<DataType>(_dim, _m, _nsc, _os, _k, verbose) {}
    virtual ~SCQuantizer() {}

    void calc_residual_vector(bool) {
        for (int k0 = 0; k0 < this->k; k0++) {
            const int bs = this->dim / this->part, kk = this->kc[k0];
            for (int i = 0; i < this->N; i++) {
                float *x = this->data + (size_t)i * this->dim;
                const float *c = this->cq[k0];
                for (int j = 0; j < this->part; j++) {
                    float d = FLT_MAX, d2 = FLT_MAX;
                    int pos = 0, pos2 = 0;
                    for (int k1 = 0; k1 < kk; k1++) {
                        const float dt = (float)distance_l2_square(x, c + (size_t)k1 * bs, bs);
                        if (d > dt) {
                            d2 = d;
                            d = dt;
                            pos2 = pos;
                            pos = k1;
                        } else if (d2 > dt) {
                            d2 = dt;
                            pos2 = k1;
                        }
                    }
                    const float *cc = c + (size_t)pos2 * bs;
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
