/*
 * bpmax_gpu.h -- C ABI of the B200 (sm_100a) BPMax fill engine, libbpmax_gpu.so.
 *
 * Plain pointers and sizes only. Every entry point returns a bpmax_status; on failure
 * bpmax_gpu_last_error() gives a message. A context owns one CUDA device, one stream and its
 * device buffers; use one context per host thread.
 *
 * Reference interface replaced (paths relative to the reference project root, with
 * V3 = TPDS/source/release/MPT_RT_V3/bpmax_complete_otf_ftable/src):
 *   void bpmax(long M, long N, long N_sec, long N_tile, long R, long MR, long NR, long P,
 *              int* seq1, int* seq2, float****** FTable)                     V3/bpmax.c:129
 * The C++ symbol itself is exported by libbpmax_gpu.so too (bpmax_b200/csrc/bpmax_shim.cpp),
 * so the reference's CLI wrapper V3/bpmax-wrapper.c links against this library unchanged.
 *
 * Sequences are int arrays of bases 0..3 = A,C,G,U (4 = any other letter), the encoding of
 * toNum in V3/external_functions.c:70-85. Strand 2 is consumed reversed, as in the reference.
 * Weights are a 12-entry table: intra-strand AU,UA,GC,CG,GU,UG then inter-strand
 * AU,UA,GC,CG,GU,UG; every weight must be finite and >= +0. The reference's hard-coded values
 * (V3/external_functions.c:58-68) are AU=UA=1.0, GC=CG=3, GU=UG=1.5 on both strands.
 */
#ifndef BPMAX_GPU_H
#define BPMAX_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

typedef enum bpmax_status {
    BPMAX_OK = 0,
    BPMAX_EINVAL = 1,   /* invalid argument (the reference prints and calls exit(-1)) */
    BPMAX_ENOMEM = 2,   /* device or pinned host allocation failed */
    BPMAX_ECUDA = 3,    /* a CUDA call failed */
    BPMAX_ENODEV = 4,   /* no CUDA device, or the kernels were not built for it */
    BPMAX_ETIMEOUT = 5  /* a device-side bounded wait gave up; the context stays usable */
} bpmax_status;

typedef struct bpmax_ctx bpmax_ctx;

/* Context life cycle. device = CUDA ordinal. */
int bpmax_gpu_create(int device, bpmax_ctx **out);
void bpmax_gpu_destroy(bpmax_ctx *ctx);
const char *bpmax_gpu_last_error(const bpmax_ctx *ctx);
const char *bpmax_gpu_status_string(int status);

/* Score weights used by later calls (default: the reference's values).
 * Replaces the link-time hook e_intra_score/e_inter_score, V3/external_functions.c:58-68. */
int bpmax_gpu_set_weights(bpmax_ctx *ctx, const float *weights12);

/* Weights of the drop-in bpmax() symbol this library exports (the reference's C++ entry point,
 * V3/bpmax.c:129). The reference reads its weights through the link-time hooks
 * e_intra_score/e_inter_score (V3/external_functions.c:58-68), which a library cannot see; this
 * sets the weights every later bpmax() call of the process uses (12 entries as above; default:
 * the reference's hard-coded values). EINVAL for a NULL pointer or a weight that is not finite
 * and >= +0, leaving the previous weights in place. Thread-safe. */
int bpmax_gpu_shim_set_weights(const float *weights12);

/* Fill of one pair into the reference's linear F layout, host memory:
 * F_lin = &FTable[0][0][0][0][0][0] of a float[M][M][N_sec][N_sec][N_tile+1][N_tile] buffer,
 * N_sec = ceil(N/N_tile), R = (N_tile - N % N_tile) % N_tile, logical cell
 * (i1,j1,i2,j2) at [i1][j1][(i2+R)/N_tile][(j2+R)/N_tile][(i2+R)%N_tile][(j2+R)%N_tile]
 * (V3/bpmax-wrapper.c:44, :175-197). Writes exactly the cells the reference fill writes
 * (logical cells, -FLT_MAX below the diagonal of diagonal tiles and in their halo row, and the
 * halo row of off-diagonal tiles = row 0 of the tile below). Cells the reference leaves
 * unwritten inside outer cells i1<=j1 (tiles with I2>J2, padding rows and columns) receive NaN;
 * outer cells i1>j1 are not touched. The table is copied out while the fill runs. With F_lin
 * pinned (cudaHostAlloc) and N <= 64, the fill also writes each cell in the reference layout into a
 * device buffer of the table's size, kept by the context for later calls (freed by
 * bpmax_gpu_destroy), and one strided copy per outer diagonal moves it to F_lin; without device
 * memory for it, or with N > 64, conversion launches per diagonal do it. A pageable F_lin is filled
 * row by row through pinned staging buffers.
 * score (may be NULL) receives F(0,M-1,0,N-1). Preconditions as the reference
 * (V3/bpmax.c:131): M>=1, N>=8, N_tile>=4, N_sec>=2, 0<=R<N_tile.
 * Replaces V3/bpmax.c:129 (the tiling arguments MR, NR, P only tune the CPU code). */
int bpmax_gpu_fill(bpmax_ctx *ctx, const int *seq1, long M, const int *seq2, long N, long N_tile,
                   float *F_lin, float *score);

/* Fill of one pair into the compact layout, host memory: T(M)=M(M+1)/2 outer cells in
 * row-major upper-triangle order, each an N x N inner table [i2][j2]; cells with i2>j2 are
 * -FLT_MAX. Same logical values as bpmax_gpu_fill. F_compact may be NULL (score only). */
int bpmax_gpu_fill_compact(bpmax_ctx *ctx, const int *seq1, long M, const int *seq2, long N,
                           float *F_compact, float *score);

/* R0-only double max-plus microbenchmark on the fill's own product kernels. Replaces the
 * reference's IPDPSW R0-only program ospsqmax_float(M, N, seq1, seq2, FTable)
 * (IPDPSW/source/R0/ospsq_coarse_diag_top_down/src/ospsqmax_float.c:113, spec ospsq_float.ab:1-15):
 *   F(i1,i1,i2,j2) = seq2[i2];  F(i1,j1,i2,i2) = seq1[i1] (j1 > i1);
 *   F(i1,j1,i2,j2) = max_{i1<=k1<j1, i2<=k2<j2} F(i1,k1,i2,k2) + F(k1+1,j1,k2+1,j2)  (j1 > i1, j2 > i2)
 * seq1[M], seq2[N]: non-negative integers (converted to float; negative values return EINVAL);
 * M >= 2, N >= 2 as the reference requires. F_compact (may be NULL) receives the compact layout of
 * bpmax_gpu_fill_compact (-FLT_MAX where i2 > j2); score (may be NULL) receives F(0,M-1,0,N-1), the
 * value the reference's program prints. Timing: bpmax_gpu_last_timing. */
int bpmax_gpu_r0_only(bpmax_ctx *ctx, const int *seq1, long M, const int *seq2, long N, float *F_compact,
                      float *score);

/* Optimal score F(0,M-1,0,N-1) of one pair, the value V3/bpmax-wrapper.c:281 prints. */
int bpmax_gpu_score(bpmax_ctx *ctx, const int *seq1, long M, const int *seq2, long N, float *score);

/* Scores of many pairs of uneven lengths in one batched fill (no reference counterpart: the
 * reference fills one pair per process run). seq1s/seq2s: per-pair host pointers; M>=1, N>=1
 * per pair. scores: num_pairs floats. */
int bpmax_gpu_score_batch(bpmax_ctx *ctx, int num_pairs, const int *const *seq1s, const long *Ms,
                          const int *const *seq2s, const long *Ns, float *scores);

/* Same pairs, one fill launch sequence per pair (the baseline the batched fill is compared to). */
int bpmax_gpu_score_each(bpmax_ctx *ctx, int num_pairs, const int *const *seq1s, const long *Ms,
                         const int *const *seq2s, const long *Ns, float *scores);

/* Forward fill plus adjoint (backward) pass of many pairs: grads[12*p + t] = d score_p / d w_t,
 * the number of times weight t is used by the optimal structure of pair p, found by following
 * argmax edges with the reference's tie-break (the later candidate of __max_float(x,y) =
 * x>y?x:y wins a tie, V3/bpmax_verify.c:576 order; the last k wins inside a reduction). No
 * reference counterpart: the reference has neither traceback nor weights as parameters. */
int bpmax_gpu_grad_batch(bpmax_ctx *ctx, int num_pairs, const int *const *seq1s, const long *Ms,
                         const int *const *seq2s, const long *Ns, float *scores, float *grads);

/* Schedule tunables of later fills (no reference counterpart: the reference's tuning knobs are its
 * compile-time tile sizes and the MR/NR/P arguments of bpmax(), V3/bpmax.c:129).
 *   BPMAX_TUNE_R0_PAIRS_PER_JOB  upper bound of k1 offset pairs (w, d-1-w) per product job (>= 1)
 *   BPMAX_TUNE_R0_MERGE_ITEMS    cost of one job's merge, in items, used to size the jobs of a diagonal
 *   BPMAX_TUNE_CLASS_STREAMS     1: width classes of a batch run as parallel graph branches; 0: one chain
 *   BPMAX_TUNE_WAIT_LIMIT_US     how long one device-side wait of a product kernel for its operand
 *                                copies may last before the kernel gives up and the call returns
 *                                BPMAX_ETIMEOUT (microseconds, 1 .. 600e6; default 4e6 = 4 s)
 *   BPMAX_TUNE_INJECT_WAIT_TIMEOUT  1: the next fill call (only that one) runs its product kernels
 *                                without issuing any operand copy, so their first waits run out with
 *                                no copy in flight; the call returns BPMAX_ETIMEOUT and later calls
 *                                are unaffected. A test of the timeout path; 0 otherwise.
 *   BPMAX_TUNE_WIDE_STAGES       shared-memory stages of the product kernel for strand-2 lengths 65..320
 *                                (2: three CTAs per SM; 3: two CTAs per SM with a deeper copy ring)
 *   BPMAX_TUNE_R0_VARIANT        shape of the product kernel for strand-2 lengths <= 64 (0: three CTAs
 *                                per SM, 168 registers, 2-4 stages; 1: two CTAs per SM, up to 255
 *                                registers, up to 6 stages)
 *   BPMAX_TUNE_CLASS_SHARE       1: with class streams, each width class's product launches take at
 *                                most its share of the SMs (its share of the padded work, at least
 *                                1/16), so the classes' chains progress side by side; 0: every launch
 *                                may take every SM
 *   BPMAX_TUNE_PERSISTENT        1 or 2: fills whose strand-2 lengths are all <= 64 run as ONE
 *                                persistent launch per width class that walks the outer diagonals as a
 *                                wavefront with device-side dependency counters (bounded waits); with
 *                                several width classes, 1 runs them side by side (each on its share of
 *                                the SMs), 2 one after another (each on every SM); 0: a graph of two
 *                                launches per outer diagonal. The R0-only mode and bpmax_gpu_fill's
 *                                per-diagonal copy-out keep the graph. */
enum bpmax_tuning_key {
    BPMAX_TUNE_R0_PAIRS_PER_JOB = 0,
    BPMAX_TUNE_R0_MERGE_ITEMS = 1,
    BPMAX_TUNE_CLASS_STREAMS = 2,
    BPMAX_TUNE_WAIT_LIMIT_US = 3,
    BPMAX_TUNE_INJECT_WAIT_TIMEOUT = 4,
    BPMAX_TUNE_WIDE_STAGES = 5,
    BPMAX_TUNE_R0_VARIANT = 6,
    BPMAX_TUNE_CLASS_SHARE = 7,
    BPMAX_TUNE_PERSISTENT = 8
};
int bpmax_gpu_set_tuning(bpmax_ctx *ctx, int key, long value);
int bpmax_gpu_get_tuning(const bpmax_ctx *ctx, int key, long *value);

/* Autotuner: fills the given pairs under candidate settings of the schedule tunables, timing
 * `trials` graph replays of each after one capture run, and keeps the fastest setting for these
 * shapes: later fills of the same shapes use it. It first tries every combination of pairs per job
 * (8 / 32 / unbounded), merge cost (1 / 4) and class streams (on / off, when the batch has several
 * width classes) with the default kernel shapes, then, on the best of those, the other product
 * kernel shape (BPMAX_TUNE_R0_VARIANT 1, when a strand-2 length is <= 64) and the deeper tile ring
 * (BPMAX_TUNE_WIDE_STAGES 3, when one is in 65..320), after trying class shares
 * (BPMAX_TUNE_CLASS_SHARE 1, when class streams won with several width classes), then the persistent
 * fill with each pairs-per-job candidate (BPMAX_TUNE_PERSISTENT 1, or 2 with several width classes,
 * when every strand-2 length is <= 64).
 * best (may be NULL) receives the 7 chosen values of keys 0, 1, 2, 6, 5, 7, 8 in that order; best_ms (may be NULL) the fill time in ms. Results of every
 * fill are unchanged by any setting (bit for bit). The reference's counterpart is choosing its tile
 * arguments N_tile, MR, NR by hand (V3/bpmax.c:129). */
int bpmax_gpu_autotune(bpmax_ctx *ctx, int num_pairs, const int *const *seq1s, const long *Ms,
                       const int *const *seq2s, const long *Ns, int trials, long *best, float *best_ms);

/* Copies part of the last fill's table to host memory: the inner tables of the outer cells (i1, j1)
 * with i1 in [i1_lo, i1_hi) and j1 in [j1_lo, j1_hi) of pair `pair` of that fill (0 for a single
 * pair), as out[i1 - i1_lo][j1 - j1_lo][N][N] floats, [i2][j2] over the reversed strand 2 as in
 * bpmax_gpu_fill_compact; -FLT_MAX where i2 > j2 and NaN for outer cells with i1 > j1. Lets a
 * caller read a window of a table too large to copy whole (no reference counterpart: the
 * reference's caller owns the whole table in host memory, V3/bpmax-wrapper.c:175-197). */
int bpmax_gpu_read_cells(bpmax_ctx *ctx, int pair, long i1_lo, long i1_hi, long j1_lo, long j1_hi, float *out);

/* Device time in milliseconds of the last fill call's kernels (CUDA events on the context's
 * stream), and the number of kernel launches it issued. */
int bpmax_gpu_last_timing(const bpmax_ctx *ctx, float *fill_ms, long *launches);

/* Re-runs the last fill's kernels one launch at a time with CUDA events around each launch on
 * the context's stream. Per kernel kind k (0 single-strand, 1 R0+R3+R4 product, 2 finalize /
 * inner wavefront): ms[k] = summed launch durations, launches[k] = launch count, terms[k] =
 * algorithmic max-plus candidates (one fp32 add + one max each) the kind evaluates (after
 * bpmax_gpu_r0_only: C(M)C(N) for kind 1, 0 for the others). Arrays of 3.
 * No reference counterpart (measurement only). */
int bpmax_gpu_profile_kernels(bpmax_ctx *ctx, float *ms, long *launches, double *terms);

/* Measured max-plus issue ceiling of this GPU: a register-resident kernel that runs the
 * instruction mix of the product kernel's inner loop (one packed fp32 add making two candidates,
 * one 3-input max merging them; every candidate a new sum, no memory traffic) on every SM.
 * terms_per_s receives candidates per second. No reference counterpart. */
int bpmax_gpu_maxplus_peak(bpmax_ctx *ctx, double *terms_per_s);

/* Score of one pair without allocating any memory. No counterpart in the reference: it serves
 * callers that cannot call cudaMalloc -- code running inside another framework's memory pool
 * or under a fixed device-memory budget, and latency-critical callers that must not risk the
 * device synchronisation cudaMalloc/cudaFree may imply. Needs no context.
 *   seq1[M], seq2[N], weights12[12]: host memory, same meaning as above; score: host float.
 *   stream: the caller's cudaStream_t (NULL = default stream); the call synchronises it.
 * All scratch lives in one fixed 64 MiB device array inside the library, which every GPU that
 * loads the library holds until the process exits. Limits: N <= 64 and, in bytes,
 * T(M)*cell + 4*M^2 + 16*M*ceil(M/2) + (a few KiB) <= 64 MiB, with T(M) = M(M+1)/2 and cell the
 * stored size of one inner table (10080 bytes at N=64, 2864 at N=32, 304 at N<=8): at most
 * M=114 for N=64, M=215 for N=32, M=654 for N<=8; larger pairs return BPMAX_EINVAL. The first
 * call on a device looks up the array's device address and sets kernel attributes for that
 * device (make it before any stream capture). Every call reuses the same array, so calls that overlap on the GPU (other threads,
 * other streams) race and must be serialised by the caller. Errors are returned as status codes
 * only (there is no context to hold a message); a CUDA error already pending on the calling thread
 * when the call starts is left in place and reported as BPMAX_ECUDA. */
int bpmax_gpu_score_noalloc(const int *seq1, long M, const int *seq2, long N, const float *weights12,
                            float *score, void *stream);

#ifdef __cplusplus
}
#endif
#endif
