/*
 * sc_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement, in plain C, of the search path of marker68/second-candidate
 * (the reference).  It is the checker for the CUDA library: only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg may load it, and
 * only to compare against or to time beside the GPU path.  The product
 * (libscgpu.so) never calls it.
 *
 * Every function cites the reference file:line it restates.  Parity of this
 * restatement with the reference itself is pinned by tests that run the
 * reference's own headers compiled by oracle/Makefile (oracle/_ref) and by the
 * golden vectors in tests/golden/ that were produced by that build.
 *
 * Floating-point conventions (identical to the reference compiled for x86-64
 * without -ffast-math and without FMA): every dot product and norm is a
 * sequential float loop "s += x[i]*y[i]" (multiply rounded, then add
 * rounded); BLAS sdot is taken to be that sequential loop.
 */
#ifndef SC_ORACLE_H_
#define SC_ORACLE_H_

#ifdef __cplusplus
extern "C" {
#endif

/* One index as the reference holds it (query.h:45-61). */
typedef struct {
    int dim, mc, kc, mp, kp, N;
    const float *cq;            /* [mc][kc][dim/mc]                          */
    const float *pq;            /* [mp][kp][dim/mp]                          */
    const float *norm_c;        /* [mc*kc]        from orc_pre_compute1      */
    const float *norm_r;        /* [mp*kp]                                   */
    const float *dot_cr;        /* [mc][kc][mp/mc][kp]                       */
    const int *L;               /* inclusive prefix counts, one per cell     */
    const int *pid;             /* [N] in cell order                         */
    const unsigned char *codes; /* [N][mp] in cell order                     */
    const float *raw;           /* [N][dim] raw vectors, or NULL             */
} orc_index;

enum { ORC_IVFADC = 0, ORC_IMI = 1, ORC_SC = 2, ORC_SC3 = 3 };
enum { ORC_ORDER_HEAP = 0, ORC_ORDER_EXACT = 1 };

void orc_pre_compute1(int dim, int mc, int kc, int mp, int kp,
                      const float *cq, const float *pq,
                      float *norm_c, float *norm_r, float *dot_cr);

void orc_pre_compute2(int dim, int mc, int kc, int mp, int kp,
                      const float *cq, const float *pq,
                      const float *norm_c, const float *norm_r,
                      const float *q, float *diff_qc, float *diff_qr);

int orc_search(const orc_index *ix, int mode, int order, const float *q,
               int w, int T, int real_dist,
               float *dist, int *ids, int cap,
               int *cells, int cap_cells, int *ncells_out,
               int *sum_out, int *empty_out);

/* The largest coarse-list rank the last orc_search popped (empty cells
 * included; -1 for IVFADC). */
int orc_last_max_rank(void);

/* Rank limit of the IMI and second-candidate walks (0 = all ranks). */
void orc_set_rank_limit(int M);

void orc_topk(const float *dist, const int *ids, int n, int R,
              float *out_d, int *out_i);

void orc_encode(int dim, int mc, int kc, int mp, int kp,
                const float *cq, const float *pq, const float *X, long n,
                unsigned short *cid, unsigned char *codes);

void orc_sc_encode(int dim, int kc, int mp, int kp, int nc,
                   const float *cq, const float *pq, const float *X, long n,
                   unsigned short *cid, unsigned char *codes);

int orc_distribution(int mode, int kc, int mc, int nc, int mp, long n,
                     const unsigned short *cid, const unsigned char *codes,
                     int *L, int *pid, unsigned char *codes_out);

double orc_distance_l2_square(const float *x, const float *y, int d);

/* Shortlist re-rank: the exact distance of each of the L ids (ids < 0 are
 * skipped) as the reference's real_dist branch computes it
 * (query.h:307-312, multi_query.h:255-259, sc_query.h:232-236: the float of
 * distance_l2_square against raw[id]), then the R smallest in (distance, id)
 * order.  Returns the number written (<= R). */
int orc_rerank(const float *raw, int dim, const float *q, const int *ids, int L, int R,
               int *out_ids, float *out_d);

#ifdef __cplusplus
}
#endif
#endif
