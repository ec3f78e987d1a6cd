/*
 * encoder.h -- drop-in for the reference's Encoder (include/encoder.h:30-60):
 * encode<T> runs the library's exact GPU encoder (codes identical to
 * encoder.h:69-192), distribution buckets rows by cell in row order
 * (encoder.cpp:170-205) and output writes the same .edat_ file
 * (encoder.cpp:207-305), with 64-bit offsets.
 */
#ifndef SCG_DROPIN_ENCODER_H_
#define SCG_DROPIN_ENCODER_H_

#include <cmath>
#include <cstdio>

#include "bucket.h"
#include "sc_utilities.h"

namespace SC {

class Encoder {
protected:
    scg_index *h = nullptr;
    PQConfig config;
    int size = 0;
    int non_empty_bucket = 0;
    int nparts_ = 0;                     // coarse ids per row (mc, or nc)
    std::vector<unsigned short> cid_;    // [N][nparts_]
    std::vector<unsigned char> codes_;   // [N][mp]
    std::vector<long long> start_;       // CSR after distribution(): cell starts
    std::vector<int> order_;             // rows in cell order

    int cells() const { return size; }

    void bucket(const std::vector<long long> &cell_of_row) {
        std::vector<long long> cnt((size_t)cells() + 1, 0);
        for (long long c : cell_of_row) cnt[(size_t)c + 1]++;
        non_empty_bucket = 0;
        for (int c = 0; c < cells(); c++) non_empty_bucket += cnt[(size_t)c + 1] > 0;
        for (int c = 0; c < cells(); c++) cnt[(size_t)c + 1] += cnt[(size_t)c];
        start_ = cnt;
        order_.assign(cell_of_row.size(), 0);
        std::vector<long long> cur(cnt.begin(), cnt.end() - 1);
        for (size_t r = 0; r < cell_of_row.size(); r++) order_[(size_t)cur[(size_t)cell_of_row[r]]++] = (int)r;
    }

    void write_edat(const char *fname) {
        FILE *f = fopen(fname, "wb");
        if (!f) {
            std::cerr << "Cannot open the file " << fname << std::endl;
            exit(1);
        }
        int hdr[2] = {non_empty_bucket, config.N};
        fwrite(hdr, sizeof(int), 2, f);
        for (int c = 0; c < cells(); c++) {
            int l = (int)(start_[(size_t)c + 1] - start_[(size_t)c]);
            fwrite(&l, sizeof(int), 1, f);
            for (long long i = start_[(size_t)c]; i < start_[(size_t)c + 1]; i++) fwrite(&order_[(size_t)i], sizeof(int), 1, f);
            for (long long i = start_[(size_t)c]; i < start_[(size_t)c + 1]; i++)
                fwrite(&codes_[(size_t)order_[(size_t)i] * config.mp], 1, (size_t)config.mp, f);
        }
        fclose(f);
    }

public:
    Encoder() {
        memset(&config, 0, sizeof(config));
        if (scg_index_create(&h, 0) != SCG_OK) scg_die("cannot create the GPU index");
    }
    virtual ~Encoder() { scg_index_destroy(h); }

    /* Encoder::load_codebooks (encoder.cpp:44-55). */
    void load_codebooks(const char *cq_path, const char *pq_path, bool verbose) {
        if (scg_load_codebooks_file(h, cq_path, pq_path) != SCG_OK) scg_die("Cannot load the codebooks");
        int64_t n = 0;
        scg_index_info(h, &config.dim, &config.mc, &config.kc, &config.mp, &config.kp, &n);
        size = (int)std::pow((double)config.kc, (double)config.mc);
        nparts_ = config.mc;
        if (verbose) std::cout << "The size of ivf:" << size << std::endl;
        std::cout << "--> Settings: (kc,mc,kp,mp)=" << config.kc << " " << config.mc << " " << config.kp << " "
                  << config.mp << std::endl;
    }

    /* Encoder::encode<T> (encoder.h:69-192). */
    template <typename DataType>
    void encode(const char *filename, int offset, bool verbose) {
        float *data = nullptr;
        config.N = load_and_convert_data<DataType, float>(filename, data, offset, config.dim, verbose);
        if (config.mc <= 0 || config.mp <= 0) {
            std::cerr << "Nothing to do" << std::endl;
            return;
        }
        cid_.assign((size_t)config.N * nparts_, 0);
        codes_.assign((size_t)config.N * config.mp, 0);
        if (encode_rows(data) != SCG_OK) scg_die("encode");
        ::operator delete(data);
    }

    /* Encoder::distribution (encoder.cpp:170-205): cell = vector_base(cid). */
    void distribution(bool verbose) {
        std::vector<long long> cell((size_t)config.N);
        for (size_t r = 0; r < cell.size(); r++) {
            long long c = 0;
            for (int j = 0; j < nparts_; j++) c = c * config.kc + cid_[r * nparts_ + j];
            cell[r] = c;
        }
        bucket(cell);
        if (verbose) std::cout << "The number of non-empty buckets: " << non_empty_bucket << std::endl;
    }

    /* Encoder::output (encoder.cpp:207-305): <db_path>/<db_prefix>_ivf.edat_ */
    void output(const char *db_path, const char *db_prefix, bool verbose) {
        char fname[512];
        snprintf(fname, sizeof(fname), "%s/%s_ivf.edat_", db_path, db_prefix);
        write_edat(fname);
        if (verbose) std::cout << "Wrote " << fname << std::endl;
    }

    PQConfig get_config() { return config; }
    const std::vector<unsigned short> &cid() const { return cid_; }
    const std::vector<unsigned char> &codes() const { return codes_; }

protected:
    virtual int encode_rows(const float *data) {
        return scg_encode(h, data, config.N, cid_.data(), codes_.data());
    }
};

}  // namespace SC
#endif
