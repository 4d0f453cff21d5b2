/*
 * bpmax_oracle.c -- CPU restatement of the BPMax recurrence (TEST INFRASTRUCTURE ONLY).
 *
 * Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker.
 * The product library never links or calls it. See bpmax_oracle.h for the layout and the
 * reference lines each function follows.
 */
#include "bpmax_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* __max_float of the reference (V3/bpmax_verify.c, "function for float max"): on a tie the
 * SECOND operand is returned. */
static inline float max_r(float x, float y) { return x > y ? x : y; }

int oracle_pair_type(int a, int b)
{
    /* V3/external_functions.c:21-39: (A,U)/(U,A) -> AU weight, (C,G)/(G,C) -> 3,
     * (G,U)/(U,G) -> GU weight. The 12-entry table splits each into its two orders. */
    if (a == 0 && b == 3) return 0; /* AU */
    if (a == 3 && b == 0) return 1; /* UA */
    if (a == 2 && b == 1) return 2; /* GC */
    if (a == 1 && b == 2) return 3; /* CG */
    if (a == 2 && b == 3) return 4; /* GU */
    if (a == 3 && b == 2) return 5; /* UG */
    return -1;
}

static inline float score6(const float *w6, int a, int b)
{
    int t = oracle_pair_type(a, b);
    return t < 0 ? 0.0f : w6[t];
}

long oracle_cell(long M, long i1, long j1) { return i1 * M - i1 * (i1 - 1) / 2 + (j1 - i1); }

void oracle_single_strand(long L, const int *s, const float *w6, float *S)
{
    /* eval_S1: S(i,j) = (i >= j-3) ? 0 : max(S(i+1,j-1) + intra(s[i],s[j]),
     *                                       max_{i<=k<j} S(i,k) + S(k+1,j)) */
    for (long i = L - 1; i >= 0; --i) {
        for (long j = i; j < L; ++j) {
            float v;
            if (i >= j - 3) {
                v = 0.0f;
            } else {
                float red = -FLT_MAX;
                for (long k = i; k < j; ++k) red = max_r(red, S[i * L + k] + S[(k + 1) * L + j]);
                v = max_r(S[(i + 1) * L + (j - 1)] + score6(w6, s[i], s[j]), red);
            }
            S[i * L + j] = v;
        }
    }
}

static int weights_ok(const float *w12)
{
    for (int t = 0; t < 12; ++t) {
        float w = w12[t];
        if (!isfinite(w) || w < 0.0f || signbit(w)) return 0;
    }
    return 1;
}

int oracle_fill(long M, long N, const int *seq1, const int *seq2, const float *w12,
                float *F, float *S1, float *S2)
{
    if (M < 1 || N < 1 || !seq1 || !seq2 || !w12 || !F || !S1 || !S2) return -1;
    if (!weights_ok(w12)) return -1;
    const float *wi = w12, *we = w12 + 6;
    const long NN = N * N;

    int *s2r = (int *)malloc(sizeof(int) * N);
    float *outer = (float *)malloc(sizeof(float) * N); /* SW1,S1+S2,R0,R3,R4 of one row */
    float *r0 = (float *)malloc(sizeof(float) * N);
    float *r2 = (float *)malloc(sizeof(float) * N);
    float *r3 = (float *)malloc(sizeof(float) * N);
    float *r4 = (float *)malloc(sizeof(float) * N);
    if (!s2r || !outer || !r0 || !r2 || !r3 || !r4) {
        free(s2r); free(outer); free(r0); free(r2); free(r3); free(r4);
        return -1;
    }
    /* strand 2 is consumed reversed: bpmax_verify.c:576 uses seq2(-i2+N-1) */
    for (long i = 0; i < N; ++i) s2r[i] = seq2[N - 1 - i];
    oracle_single_strand(M, seq1, wi, S1);
    oracle_single_strand(N, s2r, wi, S2);
    (void)outer;

    for (long i1 = M - 1; i1 >= 0; --i1) {
        for (long j1 = i1; j1 < M; ++j1) {
            float *C = F + oracle_cell(M, i1, j1) * NN;
            const long d1 = j1 - i1;
            const float s1v = S1[i1 * M + j1];
            const float w1 = d1 >= 4 ? score6(wi, seq1[i1], seq1[j1]) : 0.0f;
            const float *SW = d1 >= 4 ? F + oracle_cell(M, i1 + 1, j1 - 1) * NN : NULL;
            for (long i2 = N - 1; i2 >= 0; --i2) {
                for (long j2 = 0; j2 < i2; ++j2) C[i2 * N + j2] = -FLT_MAX;
                /* R0 row (bpmax_verify.c:584-600), vectorised over j2: for every k1, k2 the
                 * candidate F(i1,k1,i2,k2) + F(k1+1,j1,k2+1,j2) for all j2 > k2. */
                for (long j2 = i2; j2 < N; ++j2) { r0[j2] = -FLT_MAX; r3[j2] = -FLT_MAX; r4[j2] = -FLT_MAX; r2[j2] = -FLT_MAX; }
                for (long k1 = i1; k1 < j1; ++k1) {
                    const float *A = F + oracle_cell(M, i1, k1) * NN + i2 * N;
                    const float *B = F + oracle_cell(M, k1 + 1, j1) * NN;
                    for (long k2 = i2; k2 < N - 1; ++k2) {
                        const float a = A[k2];
                        const float *Bk = B + (k2 + 1) * N;
                        for (long j2 = k2 + 1; j2 < N; ++j2) r0[j2] = max_r(r0[j2], a + Bk[j2]);
                    }
                    /* R3 (:668-694): S1(i1,k1) + F(k1+1,j1,i2,j2);
                     * R4 (:695-721): F(i1,k1,i2,j2) + S1(k1+1,j1) */
                    const float s1a = S1[i1 * M + k1], s1b = S1[(k1 + 1) * M + j1];
                    const float *Brow = B + i2 * N;
                    for (long j2 = i2; j2 < N; ++j2) {
                        r3[j2] = max_r(r3[j2], s1a + Brow[j2]);
                        r4[j2] = max_r(r4[j2], A[j2] + s1b);
                    }
                }
                /* R2 (:641-667): S2(i2,k2) + F(i1,j1,k2+1,j2); rows below i2 are final. */
                for (long k2 = i2; k2 < N - 1; ++k2) {
                    const float s = S2[i2 * N + k2];
                    const float *Ck = C + (k2 + 1) * N;
                    for (long j2 = k2 + 1; j2 < N; ++j2) r2[j2] = max_r(r2[j2], s + Ck[j2]);
                }
                for (long j2 = i2; j2 < N; ++j2) {
                    const long d2 = j2 - i2;
                    float v;
                    if (d1 == 0 && d2 == 0) {
                        v = score6(we, seq1[i1], s2r[i2]); /* e_inter_score(seq1(i1),seq2(N-1-i2)) */
                    } else {
                        /* R1 (:614-640): F(i1,j1,i2,k2) + S2(k2+1,j2); same row, k2 < j2. */
                        float r1 = -FLT_MAX;
                        for (long k2 = i2; k2 < j2; ++k2) r1 = max_r(r1, C[i2 * N + k2] + S2[(k2 + 1) * N + j2]);
                        /* eval_FTable (:576): literal 0 wherever a term is undefined */
                        const float c_sw1 = d1 >= 4 ? SW[i2 * N + j2] + w1 : 0.0f;
                        const float c_sw2 = d2 >= 4 ? C[(i2 + 1) * N + (j2 - 1)] + score6(wi, s2r[i2], s2r[j2]) : 0.0f;
                        const float c_s12 = s1v + S2[i2 * N + j2];
                        const float c_r0 = (d1 >= 1 && d2 >= 1) ? r0[j2] : 0.0f;
                        const float c_r1 = d2 >= 1 ? r1 : 0.0f;
                        const float c_r2 = d2 >= 1 ? r2[j2] : 0.0f;
                        const float c_r3 = d1 >= 1 ? r3[j2] : 0.0f;
                        const float c_r4 = d1 >= 1 ? r4[j2] : 0.0f;
                        v = max_r(c_sw1, max_r(c_sw2, max_r(c_s12, max_r(c_r0, max_r(c_r1, max_r(c_r2, max_r(c_r3, c_r4)))))));
                    }
                    C[i2 * N + j2] = v;
                }
            }
        }
    }
    free(s2r); free(outer); free(r0); free(r2); free(r3); free(r4);
    return 0;
}

float oracle_score(long M, long N, const float *F)
{
    return F[oracle_cell(M, 0, M - 1) * N * N + (N - 1)];
}

/* ---------------------------------------------------------------- traceback */

enum { NODE_F = 0, NODE_S1 = 1, NODE_S2 = 2 };
typedef struct { int kind; int i1, j1, i2, j2; } node_t;

/* Keeps the LAST candidate that attains the maximum (right-nested __max_float). */
typedef struct { float v; int tag; int k1; int k2; } best_t;
static inline void consider(best_t *b, float v, int tag, int k1, int k2)
{
    if (!(b->v > v)) { b->v = v; b->tag = tag; b->k1 = k1; b->k2 = k2; }
}

long oracle_traceback(long M, long N, const int *seq1, const int *seq2, const float *w12,
                      const float *F, const float *S1, const float *S2, double *counts)
{
    if (M < 1 || N < 1 || !F || !counts) return -1;
    const float *wi = w12, *we = w12 + 6;
    const long NN = N * N;
    for (int t = 0; t < 12; ++t) counts[t] = 0.0;
    int *s2r = (int *)malloc(sizeof(int) * N);
    long cap = 8 * (M + N) + 64;
    node_t *stack = (node_t *)malloc(sizeof(node_t) * cap);
    if (!s2r || !stack) { free(s2r); free(stack); return -1; }
    for (long i = 0; i < N; ++i) s2r[i] = seq2[N - 1 - i];
#define FV(a, b, c, d) F[oracle_cell(M, (a), (b)) * NN + (long)(c) * N + (d)]
#define PUSH(K, A, B, C, D) do { if (sp >= cap) { visited = -1; goto done; } \
        stack[sp].kind = (K); stack[sp].i1 = (A); stack[sp].j1 = (B); stack[sp].i2 = (C); stack[sp].j2 = (D); ++sp; } while (0)
    long sp = 0, visited = 0;
    PUSH(NODE_F, 0, (int)M - 1, 0, (int)N - 1);
    while (sp > 0) {
        node_t n = stack[--sp];
        ++visited;
        if (n.kind == NODE_S1 || n.kind == NODE_S2) {
            const int *s = n.kind == NODE_S1 ? seq1 : s2r;
            const float *S = n.kind == NODE_S1 ? S1 : S2;
            const long L = n.kind == NODE_S1 ? M : N;
            int i = n.i1, j = n.j1;
            if (i >= j - 3) continue; /* literal 0: no pair */
            best_t b = { -FLT_MAX, -1, 0, 0 };
            consider(&b, S[(i + 1) * L + (j - 1)] + score6(wi, s[i], s[j]), 0, 0, 0);
            /* the reduction is one operand: its own last-k argmax, then compared as a unit */
            best_t r = { -FLT_MAX, -1, 0, 0 };
            for (int k = i; k < j; ++k) consider(&r, S[i * L + k] + S[(k + 1) * L + j], 1, k, 0);
            consider(&b, r.v, 1, r.k1, 0);
            if (b.tag == 0) {
                int t = oracle_pair_type(s[i], s[j]);
                if (t >= 0) counts[t] += 1.0;
                PUSH(n.kind, i + 1, j - 1, 0, 0);
            } else {
                PUSH(n.kind, i, b.k1, 0, 0);
                PUSH(n.kind, b.k1 + 1, j, 0, 0);
            }
            continue;
        }
        const int i1 = n.i1, j1 = n.j1, i2 = n.i2, j2 = n.j2;
        const int d1 = j1 - i1, d2 = j2 - i2;
        if (d1 == 0 && d2 == 0) {
            int t = oracle_pair_type(seq1[i1], s2r[i2]);
            if (t >= 0) counts[6 + t] += 1.0;
            (void)we;
            continue;
        }
        /* candidate tags: 0 SW1, 1 SW2, 2 S1+S2, 3 R0, 4 R1, 5 R2, 6 R3, 7 R4, 8 literal 0 */
        best_t b = { -FLT_MAX, -1, 0, 0 };
        if (d1 >= 4) consider(&b, FV(i1 + 1, j1 - 1, i2, j2) + score6(wi, seq1[i1], seq1[j1]), 0, 0, 0);
        else consider(&b, 0.0f, 8, 0, 0);
        if (d2 >= 4) consider(&b, FV(i1, j1, i2 + 1, j2 - 1) + score6(wi, s2r[i2], s2r[j2]), 1, 0, 0);
        else consider(&b, 0.0f, 8, 0, 0);
        consider(&b, S1[i1 * M + j1] + S2[i2 * N + j2], 2, 0, 0);
        if (d1 >= 1 && d2 >= 1) {
            best_t r = { -FLT_MAX, -1, 0, 0 };
            for (int k1 = i1; k1 < j1; ++k1)
                for (int k2 = i2; k2 < j2; ++k2)
                    consider(&r, FV(i1, k1, i2, k2) + FV(k1 + 1, j1, k2 + 1, j2), 3, k1, k2);
            consider(&b, r.v, 3, r.k1, r.k2);
        } else consider(&b, 0.0f, 8, 0, 0);
        if (d2 >= 1) {
            best_t r = { -FLT_MAX, -1, 0, 0 };
            for (int k2 = i2; k2 < j2; ++k2) consider(&r, FV(i1, j1, i2, k2) + S2[(k2 + 1) * N + j2], 4, 0, k2);
            consider(&b, r.v, 4, 0, r.k2);
            best_t q = { -FLT_MAX, -1, 0, 0 };
            for (int k2 = i2; k2 < j2; ++k2) consider(&q, S2[i2 * N + k2] + FV(i1, j1, k2 + 1, j2), 5, 0, k2);
            consider(&b, q.v, 5, 0, q.k2);
        } else { consider(&b, 0.0f, 8, 0, 0); consider(&b, 0.0f, 8, 0, 0); }
        if (d1 >= 1) {
            best_t r = { -FLT_MAX, -1, 0, 0 };
            for (int k1 = i1; k1 < j1; ++k1) consider(&r, S1[i1 * M + k1] + FV(k1 + 1, j1, i2, j2), 6, k1, 0);
            consider(&b, r.v, 6, r.k1, 0);
            best_t q = { -FLT_MAX, -1, 0, 0 };
            for (int k1 = i1; k1 < j1; ++k1) consider(&q, FV(i1, k1, i2, j2) + S1[(k1 + 1) * M + j1], 7, k1, 0);
            consider(&b, q.v, 7, q.k1, 0);
        } else { consider(&b, 0.0f, 8, 0, 0); consider(&b, 0.0f, 8, 0, 0); }

        switch (b.tag) {
        case 0: {
            int t = oracle_pair_type(seq1[i1], seq1[j1]);
            if (t >= 0) counts[t] += 1.0;
            PUSH(NODE_F, i1 + 1, j1 - 1, i2, j2);
        } break;
        case 1: {
            int t = oracle_pair_type(s2r[i2], s2r[j2]);
            if (t >= 0) counts[t] += 1.0;
            PUSH(NODE_F, i1, j1, i2 + 1, j2 - 1);
        } break;
        case 2: PUSH(NODE_S1, i1, j1, 0, 0); PUSH(NODE_S2, i2, j2, 0, 0); break;
        case 3: PUSH(NODE_F, i1, b.k1, i2, b.k2); PUSH(NODE_F, b.k1 + 1, j1, b.k2 + 1, j2); break;
        case 4: PUSH(NODE_F, i1, j1, i2, b.k2); PUSH(NODE_S2, b.k2 + 1, j2, 0, 0); break;
        case 5: PUSH(NODE_S2, i2, b.k2, 0, 0); PUSH(NODE_F, i1, j1, b.k2 + 1, j2); break;
        case 6: PUSH(NODE_S1, i1, b.k1, 0, 0); PUSH(NODE_F, b.k1 + 1, j1, i2, j2); break;
        case 7: PUSH(NODE_F, i1, b.k1, i2, j2); PUSH(NODE_S1, b.k1 + 1, j1, 0, 0); break;
        default: break; /* literal 0: empty structure */
        }
    }
done:
#undef FV
#undef PUSH
    free(s2r);
    free(stack);
    return visited;
}

/* ---------------------------------------------------------------- reference layout */

long oracle_reference_size(long M, long N, long T)
{
    long Ns = (N + T - 1) / T;
    return M * M * Ns * Ns * (T + 1) * T;
}

void oracle_to_reference_layout(long M, long N, long T, const float *F, float *Fr)
{
    const long Ns = (N + T - 1) / T, R = (T - N % T) % T, NN = N * N;
    for (long i1 = 0; i1 < M; ++i1)
        for (long j1 = i1; j1 < M; ++j1) {
            const float *C = F + oracle_cell(M, i1, j1) * NN;
            for (long I2 = 0; I2 < Ns; ++I2)
                for (long J2 = I2; J2 < Ns; ++J2) {
                    float *tile = Fr + (((i1 * M + j1) * Ns + I2) * Ns + J2) * (T + 1) * T;
                    const long Ri = I2 == 0 ? R : 0, Rj = (I2 == 0 && J2 == 0) ? R : 0;
                    for (long r = Ri; r < T; ++r)
                        for (long c = Rj; c < T; ++c) {
                            const long i2 = I2 * T + r - R, j2 = J2 * T + c - R;
                            tile[r * T + c] = (i2 <= j2) ? C[i2 * N + j2] : -FLT_MAX;
                        }
                    for (long c = Rj; c < T; ++c) {
                        if (I2 == J2) tile[T * T + c] = -FLT_MAX;
                        else tile[T * T + c] = C[((I2 + 1) * T - R) * N + (J2 * T + c - R)];
                    }
                }
        }
}

int oracle_reference_written(long M, long N, long T, long idx)
{
    const long Ns = (N + T - 1) / T, R = (T - N % T) % T;
    long c = idx % T; idx /= T;
    long r = idx % (T + 1); idx /= (T + 1);
    long J2 = idx % Ns; idx /= Ns;
    long I2 = idx % Ns; idx /= Ns;
    long j1 = idx % M; idx /= M;
    long i1 = idx;
    if (i1 > j1 || I2 > J2) return 0;
    const long Ri = I2 == 0 ? R : 0, Rj = (I2 == 0 && J2 == 0) ? R : 0;
    if (c < Rj) return 0;
    if (r < T && r < Ri) return 0;
    return 1;
}

int oracle_r0only(long M, long N, const int *seq1, const int *seq2, float *F)
{
    if (M < 1 || N < 1) return -1;
    const long NN = N * N;
    for (long d1 = 0; d1 < M; ++d1)
        for (long i1 = 0; i1 + d1 < M; ++i1) {
            const long j1 = i1 + d1;
            float *C = F + oracle_cell(M, i1, j1) * NN;
            for (long q = 0; q < NN; ++q) C[q] = -FLT_MAX;
            for (long d2 = 0; d2 < N; ++d2)
                for (long i2 = 0; i2 + d2 < N; ++i2) {
                    const long j2 = i2 + d2;
                    float v;
                    if (j1 == i1) {
                        v = (float)seq2[i2];
                    } else if (j2 == i2) {
                        v = (float)seq1[i1];
                    } else {
                        v = -INFINITY;
                        for (long k1 = i1; k1 < j1; ++k1) {
                            const float *A = F + oracle_cell(M, i1, k1) * NN;
                            const float *B = F + oracle_cell(M, k1 + 1, j1) * NN;
                            for (long k2 = i2; k2 < j2; ++k2) v = max_r(v, A[i2 * N + k2] + B[(k2 + 1) * N + j2]);
                        }
                    }
                    C[i2 * N + j2] = v;
                }
        }
    return 0;
}
