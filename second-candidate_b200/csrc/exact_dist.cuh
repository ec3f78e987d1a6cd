// Exact squared distance of distance_l2_square
// (lib/simple-cluster/include/utilities.h:217-230), the arithmetic of the
// reference's real_dist branch (query.h:307-312): each difference a float
// subtraction, squared and summed in double in dimension order, the result
// stored as float.  Shared by the shortlist re-rank (rerank.cu) and the
// all-candidate exact scan (search_impl.cuh).
#pragma once

#include "scg_internal.cuh"

namespace scg {

__device__ __forceinline__ float to_f(float x) { return x; }
__device__ __forceinline__ float to_f(uint8_t x) { return (float)x; }

template <typename T>
__device__ __forceinline__ float exact_dist(const float *__restrict__ q, const T *__restrict__ x, int dim) {
    double dis = 0.0;
    for (int t = 0; t < dim; t++) {
        const double tmp = (double)__fsub_rn(q[t], to_f(__ldg(x + t)));
        dis = __dadd_rn(dis, __dmul_rn(tmp, tmp));
    }
    return (float)dis;
}

__device__ __forceinline__ void acc_sq(double &dis, float qv, float xv) {
    const double tmp = (double)__fsub_rn(qv, xv);
    dis = __dadd_rn(dis, __dmul_rn(tmp, tmp));
}

// The same sum with the row read 16 bytes at a time (rows 16-byte aligned,
// dim a multiple of 16 bytes), eight loads in flight per thread and the
// query read as float4 from shared memory: the dimension order, hence the
// value, is unchanged.
__device__ __forceinline__ float exact_dist_vec(const float *__restrict__ q, const uint8_t *__restrict__ x, int dim) {
    double dis = 0.0;
    const uint4 *xv = reinterpret_cast<const uint4 *>(x);
    const float4 *q4 = reinterpret_cast<const float4 *>(q);
    const int n = dim / 16;
    int c = 0;
    for (; c < n; c += 8) {
        uint4 v[8];
#pragma unroll
        for (int j = 0; j < 8; j++) v[j] = c + j < n ? __ldg(xv + c + j) : make_uint4(0, 0, 0, 0);
#pragma unroll
        for (int j = 0; j < 8; j++) {
            if (c + j >= n) break;
            const uint32_t w[4] = {v[j].x, v[j].y, v[j].z, v[j].w};
#pragma unroll
            for (int g = 0; g < 4; g++) {
                const float4 qq = q4[(c + j) * 4 + g];
                acc_sq(dis, qq.x, (float)(w[g] & 0xffu));
                acc_sq(dis, qq.y, (float)((w[g] >> 8) & 0xffu));
                acc_sq(dis, qq.z, (float)((w[g] >> 16) & 0xffu));
                acc_sq(dis, qq.w, (float)(w[g] >> 24));
            }
        }
    }
    return (float)dis;
}

__device__ __forceinline__ float exact_dist_vec(const float *__restrict__ q, const float *__restrict__ x, int dim) {
    double dis = 0.0;
    const float4 *xv = reinterpret_cast<const float4 *>(x);
    const float4 *q4 = reinterpret_cast<const float4 *>(q);
    const int n = dim / 4;
    for (int c = 0; c < n; c += 8) {
        float4 v[8];
#pragma unroll
        for (int j = 0; j < 8; j++) v[j] = c + j < n ? __ldg(xv + c + j) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int j = 0; j < 8; j++) {
            if (c + j >= n) break;
            const float4 qq = q4[c + j];
            acc_sq(dis, qq.x, v[j].x);
            acc_sq(dis, qq.y, v[j].y);
            acc_sq(dis, qq.z, v[j].z);
            acc_sq(dis, qq.w, v[j].w);
        }
    }
    return (float)dis;
}

// Either form for one row: 16-byte loads when the row is 16-byte aligned and
// a multiple of 16 bytes long (the value is the same).
template <typename T>
__device__ __forceinline__ float exact_dist_row(const float *__restrict__ q, const T *__restrict__ x, int dim,
                                                bool vec) {
    return vec ? exact_dist_vec(q, x, dim) : exact_dist(q, x, dim);
}

}  // namespace scg
