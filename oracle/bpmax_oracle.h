/*
 * bpmax_oracle.h -- CPU restatement of the BPMax recurrence (TEST INFRASTRUCTURE ONLY).
 *
 * This is the checker the parity tests compare the CUDA fill against. It is never linked
 * into, loaded by, or called from the product library (bpmax_b200/); only tests/, the
 * smoke entry point and bench.py's CPU-baseline leg use it.
 *
 * It restates the AlphaZ "verify" program of the reference
 *   TPDS/source/release/MPT_RT_V3/bpmax_complete_otf_ftable/src/bpmax_verify.c
 * (eval_S1 :533-544, eval_S2 :560-571, eval_FTable :572-583, R0 :584-613, R1 :614-640,
 *  R2 :641-667, R3 :668-694, R4 :695-721) as a bottom-up loop nest instead of memoised
 * recursion. Every F cell is a max over candidates that are each ONE fp32 add of two stored
 * values (or a stored value / literal 0), so the loop order does not change any bit.
 *
 * Parity pin: the restatement is checked against the reference's own bpmax_verify() and its
 * optimised bpmax() fill, both compiled from the reference sources by oracle/Makefile into
 * oracle/_ref/, and against the golden fixtures in tests/golden/ that script generated.
 *
 * Weights: a 12-entry table replaces the hard-coded score hook of the reference
 * (V3/external_functions.c:21-68): w[0..5] = intra-strand AU,UA,GC,CG,GU,UG and
 * w[6..11] = inter-strand AU,UA,GC,CG,GU,UG. Bases are 0..4 = A,C,G,U,N (toNum,
 * V3/external_functions.c:70-85); any other pair scores 0 (no_interact_value).
 * The reference's own weights are AU=UA=1.0, GC=CG=3, GU=UG=1.5 for both strands.
 */
#ifndef BPMAX_ORACLE_H
#define BPMAX_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Pair-type index 0..5 (AU,UA,GC,CG,GU,UG) for the ordered base pair (a,b), or -1. */
int oracle_pair_type(int a, int b);

/* Index of outer cell (i1,j1), i1<=j1<M, in the row-major upper triangle. */
long oracle_cell(long M, long i1, long j1);

/* Single-strand table S[i*L+j] (i<=j) of the sequence s[0..L-1] with intra weights w6.
 * Cells with i>j are left untouched. bpmax_verify.c:533-544 (S1); S2 is the same DP over
 * the reversed strand 2, bpmax_verify.c:560-571. */
void oracle_single_strand(long L, const int *s, const float *w6, float *S);

/* Full fill. F holds T(M)=M(M+1)/2 inner tables of N*N floats, cell (i1,j1) at
 * F + oracle_cell(M,i1,j1)*N*N, inner cell (i2,j2) at [i2*N+j2]; inner index i2 runs over the
 * REVERSED strand 2 (base seq2[N-1-i2]). Cells with i2>j2 are set to -FLT_MAX.
 * S1 (M*M) and S2 (N*N) receive the single-strand tables (S2 over reversed strand 2).
 * Returns 0, or -1 on invalid arguments (M<1, N<1, negative or non-finite weight). */
int oracle_fill(long M, long N, const int *seq1, const int *seq2, const float *w12,
                float *F, float *S1, float *S2);

/* Optimal score F(0,M-1,0,N-1) of a filled table. */
float oracle_score(long M, long N, const float *F);

/* Traceback of the optimum along argmax edges with the reference's tie-break: a right-nested
 * __max_float(x,y)=x>y?x:y (bpmax_verify.c:62-64 style) picks the LAST candidate that attains
 * the maximum in the order SW1,SW2,S1+S2,R0,R1,R2,R3,R4 (eval_FTable :576), and every
 * reduction keeps the LAST k attaining it (k1 outer, k2 inner for R0, :591-597).
 * counts[12] receives how many times each weight is used by the optimal structure, i.e.
 * d(score)/d(w). Returns the number of traceback nodes visited, or -1 on error. */
long oracle_traceback(long M, long N, const int *seq1, const int *seq2, const float *w12,
                      const float *F, const float *S1, const float *S2, double *counts);

/* Number of floats in the reference's linear F buffer
 * M*M*N_sec*N_sec*(N_tile+1)*N_tile (V3/bpmax-wrapper.c:175-197). */
long oracle_reference_size(long M, long N, long N_tile);

/* Writes a compact table into the reference's linear layout
 * F_ref[i1][j1][I2][J2][r][c] (V3/bpmax-wrapper.c:44), exactly the cells the reference fill
 * writes: logical cells, -FLT_MAX below the diagonal of diagonal tiles and in their halo row
 * (V3/bpmax_ftable_init.c:171-214), and the halo row of off-diagonal tiles = row 0 of the
 * tile below (V3/bpmax_inner_reductions_finalize.c:132). Padding cells and i1>j1 outer
 * cells are not touched. */
void oracle_to_reference_layout(long M, long N, long N_tile, const float *F, float *F_ref);

/* 1 if reference-layout cell (linear index idx) is one the reference fill writes, else 0. */
int oracle_reference_written(long M, long N, long N_tile, long idx);

/* R0-only double max-plus (the IPDPSW microbenchmark spec,
 * IPDPSW/source/R0/ospsq_coarse_diag_top_down/ospsq_float.ab:1-15; its C kernel is
 * IPDPSW/source/R0/ospsq_coarse_diag_top_down/src/ospsqmax_float.c:113-189):
 *   F(i1,i1,i2,j2) = seq2[i2]
 *   F(i1,j1,i2,i2) = seq1[i1]                                            (j1 > i1)
 *   F(i1,j1,i2,j2) = max_{i1<=k1<j1, i2<=k2<j2} F(i1,k1,i2,k2) + F(k1+1,j1,k2+1,j2)   (j1 > i1, j2 > i2)
 * with the integer sequences converted to float. F: compact layout as oracle_fill (T(M) cells
 * of N x N, -FLT_MAX where i2 > j2). Returns 0, or -1 for M < 1 or N < 1. */
int oracle_r0only(long M, long N, const int *seq1, const int *seq2, float *F);

#ifdef __cplusplus
}
#endif
#endif
