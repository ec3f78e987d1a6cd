/*
 * sc_encoder.h -- drop-in for the reference's SCEncoder
 * (include/sc_encoder.h:32-54): the nc nearest coarse centroids per row
 * (codes identical to sc_encoder.h:205-332), cells kc^nc keyed
 * nn1*kc + nn2 (sc_encoder.cpp:39-48), written as <prefix>_mr<nc>_ivf.edat_
 * (sc_encoder.cpp:83-182).
 */
#ifndef SCG_DROPIN_SC_ENCODER_H_
#define SCG_DROPIN_SC_ENCODER_H_

#include "encoder.h"

namespace SC {

class SCEncoder : public Encoder {
protected:
    int nc;
    int encode_rows(const float *data) override {
        return scg_sc_encode(h, data, config.N, nc, cid_.data(), codes_.data());
    }

public:
    SCEncoder() : Encoder(), nc(2) {}
    explicit SCEncoder(int n) : Encoder(), nc(n) { std::cout << "nc = " << nc << std::endl; }
    virtual ~SCEncoder() {}

    void load_codebooks(const char *cq_path, const char *pq_path, bool verbose) {
        Encoder::load_codebooks(cq_path, pq_path, verbose);
        nparts_ = nc;
        size = (int)std::pow((double)config.kc, (double)nc);
    }

    template <typename DataType>
    void encode(const char *filename, int offset, bool verbose) {
        Encoder::encode<DataType>(filename, offset, verbose);
    }

    void output(const char *db_path, const char *db_prefix, bool verbose) {
        char fname[512];
        snprintf(fname, sizeof(fname), "%s/%s_mr%d_ivf.edat_", db_path, db_prefix, nc);
        write_edat(fname);
        if (verbose) std::cout << "Wrote " << fname << std::endl;
    }
};

}  // namespace SC
#endif
