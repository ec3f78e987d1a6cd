/*
 * sc_utilities.h -- drop-in for the reference header of the same name
 * (include/sc_utilities.h): the configuration record and the TEXMEX loaders
 * the search path's callers use, over the B200 library's C ABI (scg.h).
 *
 * Errors keep the reference's behaviour: I/O failures print to cerr and end
 * the process with EXIT_FAILURE (sc_utilities.h:826-846).
 */
#ifndef SCG_DROPIN_SC_UTILITIES_H_
#define SCG_DROPIN_SC_UTILITIES_H_

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include "scg.h"

namespace SC {
typedef unsigned short ushort;

/* PQConfig, sc_utilities.h:801-805 (same fields and meaning). */
typedef struct {
    int N, kc, kp, mc, mp, w, dim, T, L;
    char db_prefix[256];
    char db_path[256];
} PQConfig;

/* Message of the last failing library call. */
inline std::string scg_message() {
    char buf[512];
    scg_last_error(buf, sizeof(buf));
    return std::string(buf);
}

/* Prints the library's message and ends the process, as the reference does
 * on I/O failures. */
inline void scg_die(const char *what) {
    std::cerr << what << ": " << scg_message() << std::endl;
    exit(EXIT_FAILURE);
}

/* Reads a TEXMEX file whose rows are a `header`-byte prefix followed by d
 * values of DataType1, converting them to DataType2.  Returns the row count.
 * Same contract as load_and_convert_data (sc_utilities.h:1078-1143): data is
 * allocated with ::operator new and freed by the caller with ::delete. */
template <typename DataType1, typename DataType2>
inline int load_and_convert_data(const char *filename, DataType2 *&data, int header, int d, bool verbose) {
    if (d <= 0 || filename == nullptr) {
        if (verbose) std::cerr << "Defective data!" << std::endl;
        exit(1);
    }
    FILE *f = fopen(filename, "rb");
    if (!f) {
        if (verbose) std::cerr << "Cannot open the file " << filename << std::endl;
        exit(1);
    }
    fseek(f, 0, SEEK_END);
    size_t size = (size_t)ftell(f);
    fseek(f, 0, SEEK_SET);
    size_t row = (size_t)d * sizeof(DataType1) + (size_t)header;
    size_t rows = size / row;
    std::vector<unsigned char> buf(row);
    data = (DataType2 *)::operator new(rows * (size_t)d * sizeof(DataType2));
    for (size_t r = 0; r < rows; r++) {
        if (fread(buf.data(), 1, row, f) != row) break;
        for (int j = 0; j < d; j++) {
            DataType1 v;
            memcpy(&v, buf.data() + header + (size_t)j * sizeof(DataType1), sizeof(DataType1));
            data[r * (size_t)d + j] = static_cast<DataType2>(v);
        }
    }
    fclose(f);
    if (verbose) std::cout << "The number of vectors: " << rows << std::endl;
    return (int)rows;
}

/* distance_l2_square (lib/simple-cluster/include/utilities.h:217-230):
 * float differences, squared and summed in double. */
template <typename DataType1, typename DataType2>
inline double distance_l2_square(const DataType1 *x, const DataType2 *y, int d) {
    double dis = 0.0, tmp;
    for (int i = 0; i < d; i++) {
        tmp = static_cast<float>(x[i]) - static_cast<float>(y[i]);
        dis += tmp * tmp;
    }
    return dis;
}

/* load_codebook (sc_utilities.h:897-980) for the coarse (type 0) and product
 * (type 1) codebooks: the .ctr_ header {k, m, dim} fills config (kc/mc or
 * kp/mp, dim) and `codebook` receives k * dim values (::operator new). */
template <typename DataType>
inline void load_codebook(const char *filename, PQConfig &config, DataType *&codebook, int type, bool verbose) {
    FILE *f = fopen(filename, "rb");
    if (!f) {
        if (verbose) std::cerr << "Cannot open the file" << std::endl;
        exit(1);
    }
    DataType hdr[3];
    if (fread(hdr, sizeof(DataType), 3, f) != 3) {
        std::cerr << "Wrong data" << std::endl;
        exit(EXIT_FAILURE);
    }
    config.dim = static_cast<int>(hdr[2]);
    const int k = static_cast<int>(hdr[0]), m = static_cast<int>(hdr[1]);
    if (type == 1) {
        config.kp = k;
        config.mp = m;
    } else {
        config.kc = k;
        config.mc = m;
    }
    if (m == 0) {
        std::cerr << "Wrong data" << std::endl;
        exit(EXIT_FAILURE);
    }
    codebook = (DataType *)::operator new(sizeof(DataType) * (size_t)k * config.dim);
    if (fread(codebook, sizeof(DataType), (size_t)k * config.dim, f) != (size_t)k * config.dim) {
        std::cerr << "Wrong data" << std::endl;
        exit(EXIT_FAILURE);
    }
    fclose(f);
    if (verbose) std::cout << "Loaded a codebook at " << filename << " with " << m << " sub codes" << std::endl;
}

/* load_data (sc_utilities.h:817-886): no conversion. */
template <typename DataType>
inline int load_data(const char *filename, DataType *&data, int header, int d, bool verbose) {
    return load_and_convert_data<DataType, DataType>(filename, data, header, d, verbose);
}
}  // namespace SC

#endif
