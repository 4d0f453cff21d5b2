// bpmax_kernels.cuh -- sm_100a kernels of the BPMax fill.
//
// Recurrence (reference spec V3cs/bpmax_verify.ab:16-71, executed by
// V3/bpmax_verify.c:533-721; V3 = TPDS/source/release/MPT_RT_V3/bpmax_complete_otf_ftable/src):
//   F(i1,j1,i2,j2) = inter(s1[i1],s2r[i2])                            if i1==j1 && i2==j2
//                  = max( SW1, SW2, S1(i1,j1)+S2(i2,j2), R0, R1, R2, R3, R4 ) otherwise,
// each candidate one fp32 add of two stored values (or a literal 0 where undefined).
// With weights >= +0 every value is >= +0, so (a) max is exact and order-free, (b) integer
// max on the float bit patterns equals the float max, which lets partial maxima from many
// CTAs merge with atomicMax on int, and (c) masked cells can hold -inf (never a winner).
//
// Device layout of one sequence pair (a "pair" below):
//   outer cell (i1,j1), i1<=j1<M, index c = i1*M - i1*(i1-1)/2 + (j1-i1) (row-major triangle)
//   F: one inner table per outer cell, i2 over the reversed strand 2, Np = N rounded up:
//     Np <= 64 (Np = 8*NB): a "cell image" of 16-byte chunks -- block columns BJ = 0..NB-1 in
//       turn, column BJ holding the 8x8 blocks (0..BJ, BJ) of the upper block triangle at a pitch
//       of 17 chunks (row r of a block = chunks 2r, 2r+1; the 17th chunk is spare), then the
//       column's 2-chunk S1 piece (-inf x7, S1 of the cell), then R0_TAB_COLPAD[NB][BJ] spare
//       chunks (the pads spread the product kernel's shared loads over the bank groups). Inside
//       diagonal blocks the entries below the diagonal are -inf except the subdiagonal, which
//       holds S1 of the cell; padding rows/columns (>= N) are -inf.
//     64 < Np <= 320 (a multiple of 64): tile images (below);
//     Np > 320: row-major Np x Np with -inf outside the logical triangle and S1 on the
//       subdiagonal, plus FT, the same table transposed (bpmax_kernels_large.cuh).
//   S1[M][M], S2[Np][Np] single-strand tables (S2 over the reversed strand 2)
#pragma once
#include <cstdint>
#include <type_traits>
#include <cuda_runtime.h>

namespace bpmax {

constexpr float NEG_INF = -__builtin_inff();

#include "r0_tables.inc"

// chunk offset of block column c of a cell image of width class nb (c = nb: the image size)
#ifdef __CUDA_ARCH__
#define IMG_COLBASE(nb, c) c_img_colbase[nb][c]
#else
#define IMG_COLBASE(nb, c) R0_TAB_COLBASE[nb][c]
#endif

struct Weights {
    float w[12];  // intra AU,UA,GC,CG,GU,UG ; inter AU,UA,GC,CG,GU,UG
};

struct PairDesc {
    int M, N, Np;
    int cnt_off;       // persistent fill: offset of the pair's per-diagonal counters (M ints)
    long long F_off;   // float offset of F[0] (and of FT[0] in the FT arena)
    long long S1_off;  // float offset of S1 in the S arena
    long long S2_off;  // float offset of S2 in the S arena
    long long S2m_off; // Np > 64 only: S2 with -inf outside its triangle
    long long S2t_off; // Np > 64 only: ST1[j][k] = S2(k+1, j), -inf outside
    long long S2d_off; // Np > 64 only: S2 diagonal-major and triangular, S2(i, i+e) at drow(Np, e) + i, -inf outside
    int seq1_off;      // offset of seq1 in the base arena (uint8)
    int seq2_off;      // offset of the REVERSED seq2 in the base arena (uint8)
    long long cell_base;  // persistent fill: index of the pair's cell (0, 0) among all pairs' cells
};

// pair type of ordered bases (a,b): AU=0 UA=1 GC=2 CG=3 GU=4 UG=5, else -1
// (V3/external_functions.c:21-39, split by order for the 12-entry table)
__host__ __device__ __forceinline__ int pair_type(int a, int b)
{
    if ((a | b) & ~3) return -1;
    // nibble (a*4+b) -> type, F = none: idx3 -> 0 (AU), idx6 -> 3 (CG), idx9 -> 2 (GC),
    // idx11 -> 4 (GU), idx12 -> 1 (UA), idx14 -> 5 (UG)
    const uint64_t tab = 0xF5F14F2FF3FF0FFFull;
    int v = (int)((tab >> (4 * (a * 4 + b))) & 0xF);
    return v == 0xF ? -1 : v;
}

__host__ __device__ __forceinline__ float score_w(const float *w6, int a, int b)
{
    int t = pair_type(a, b);
    return t < 0 ? 0.0f : w6[t];
}

__host__ __device__ __forceinline__ long long cell_index(int M, int i1, int j1)
{
    return (long long)i1 * M - (long long)i1 * (i1 - 1) / 2 + (j1 - i1);
}

__device__ __forceinline__ float fmax3(float a, float b, float c) { return fmaxf(fmaxf(a, b), c); }

// ------------------------------------------------------------------------------------------
// Tile images: inner tables of width 64 < Np <= WIDE_TILE_MAX_NP (Np = 64 * NT) are stored per
// outer cell as the upper triangle of NT x NT tiles of 64 x 64 in row-major tile-triangle order. A
// diagonal tile is a width-64 cell image (above); an off-diagonal ("dense") tile holds all 64 of
// its 8x8 blocks in block columns at WIDE_DENSE_COLBASE (wide_tables.inc), each column closed by a
// halo piece: row 0 of block (0, bj) of the tile below, the row after the tile, so the row-shifted
// operand of any tile is one image. Rows and columns >= N are -inf.
// Wider tables (Np > WIDE_TILE_MAX_NP) are row-major with a transposed copy (bpmax_kernels_large.cuh).
// ------------------------------------------------------------------------------------------
#include "wide_tables.inc"

constexpr int WIDE_TILE_MAX_NP = 320;                     // widest table stored as tile images
constexpr int WIDE_DIAG_CHUNKS = R0_TAB_COLBASE[8][8];    // diagonal tile image (width-64 cell image)
constexpr int WIDE_DENSE_CHUNKS = WIDE_DENSE_COLBASE[8];  // dense tile image

__host__ __device__ __forceinline__ bool is_tiled(int Np) { return Np > 64 && Np <= WIDE_TILE_MAX_NP; }

// float offset of tile (I, J), I <= J, inside a cell's table of NT x NT tiles
__host__ __device__ __forceinline__ long long wide_tile_off(int NT, int I, int J)
{
    const long long SD = 4LL * WIDE_DIAG_CHUNKS, SQ = 4LL * WIDE_DENSE_CHUNKS;
    long long o = (long long)I * SD + SQ * ((long long)I * (NT - 1) - (long long)I * (I - 1) / 2);
    if (J > I) o += SD + (long long)(J - I - 1) * SQ;
    return o;
}
__host__ __device__ __forceinline__ long long wide_cell_floats(int NT)
{
    return (long long)NT * 4 * WIDE_DIAG_CHUNKS + (long long)NT * (NT - 1) / 2 * 4 * WIDE_DENSE_CHUNKS;
}

#ifdef __CUDA_ARCH__
#define WIDE_DENSE_CB(c) c_wide_dense_colbase[c]
#else
#define WIDE_DENSE_CB(c) WIDE_DENSE_COLBASE[c]
#endif

// float offset, inside a cell's table of NT x NT tiles, of the stored entry (r, c) with r <= c
__host__ __device__ __forceinline__ long long wide_pos(int NT, int r, int c)
{
    const int I = r >> 6, J = c >> 6, lr = r & 63, lc = c & 63, bi = lr >> 3, bj = lc >> 3;
    const int cb = I == J ? IMG_COLBASE(8, bj) : WIDE_DENSE_CB(bj);
    return wide_tile_off(NT, I, J) + 4 * (cb + 17 * bi) + 8 * (lr & 7) + (lc & 7);
}

// floats per stored cell table of a pair
__host__ __device__ __forceinline__ long long cell_floats(int Np)
{
    if (Np <= 64) return 4LL * IMG_COLBASE(Np >> 3, Np >> 3);
    if (Np <= WIDE_TILE_MAX_NP) return wide_cell_floats(Np >> 6);
    return (long long)Np * Np;
}

// F(cell)[r][c] for any r, c < Np (entries below the diagonal as the tables define them)
__device__ __forceinline__ float f_value(const PairDesc &pd, const float *__restrict__ F, long long cell, int r, int c)
{
    const float *C = F + pd.F_off + cell * cell_floats(pd.Np);
    if (pd.Np > WIDE_TILE_MAX_NP) return C[(long long)r * pd.Np + c];
    if (pd.Np > 64) {
        if (r > c) return r == c + 1 ? C[4 * 17 + 7] : NEG_INF;  // S1 piece of column 0 of tile (0, 0)
        return C[wide_pos(pd.Np >> 6, r, c)];
    }
    const int NB = pd.Np >> 3, BI = r >> 3, BJ = c >> 3;
    if (BI > BJ) return r == c + 1 ? C[4 * 17 + 7] : NEG_INF;  // S1 piece of column 0
    return C[4 * (c_img_colbase[NB][BJ] + 17 * BI) + 8 * (r & 7) + (c & 7)];
}

// ------------------------------------------------------------------------------------------
// Single-strand table S2 over the reversed strand 2 (V3/bpmax_verify.c:560-571):
// S(i,j) = 0 if j-i<=3, else max(S(i+1,j-1)+intra(s[i],s[j]), max_{i<=k<j} S(i,k)+S(k+1,j)).
// One CTA per pair; wavefront over the diagonal j-i. Cells outside the N x N upper triangle are
// left at 0 and never read. (S1 is built diagonal by diagonal inside finalize_small_kernel.) Pairs
// with tables wider than the tile images are left to s2_diag_kernel, one launch per diagonal.
// ------------------------------------------------------------------------------------------
__global__ void single_strand_kernel(const PairDesc *__restrict__ pairs, const uint8_t *__restrict__ bases,
                                     float *__restrict__ S, Weights W)
{
    const PairDesc pd = pairs[blockIdx.x];
    if (pd.Np > WIDE_TILE_MAX_NP) return;  // row-major tables: one launch per diagonal (s2_diag_kernel)
    const bool second = true;
    const int L = second ? pd.N : pd.M;
    const int ld = second ? pd.Np : pd.M;
    const uint8_t *s = bases + (second ? pd.seq2_off : pd.seq1_off);
    float *T = S + (second ? pd.S2_off : pd.S1_off);
    for (int idx = threadIdx.x; idx < ld * ld; idx += blockDim.x) T[idx] = 0.0f;
    __syncthreads();
    for (int d = 4; d < L; ++d) {
        const int cells = L - d;
        // groups of g threads per cell, g a power of two <= 32
        int g = 1;
        while (g < 32 && g * 2 * cells <= (int)blockDim.x) g *= 2;
        const int lane_g = threadIdx.x & (g - 1);
        const int slots = blockDim.x / g;
        for (int base = 0; base < cells; base += slots) {
            const int i = base + threadIdx.x / g;
            float red = NEG_INF;
            const bool act = i < cells;
            const int j = i + d;
            if (act)
                for (int k = i + lane_g; k < j; k += g) red = fmaxf(red, T[i * ld + k] + T[(k + 1) * ld + j]);
            for (int o = g >> 1; o > 0; o >>= 1) red = fmaxf(red, __shfl_xor_sync(0xffffffffu, red, o, g));
            if (act && lane_g == 0) {
                const float pr = T[(i + 1) * ld + (j - 1)] + score_w(W.w, s[i], s[j]);
                T[i * ld + j] = fmaxf(pr, red);
            }
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------------------------------
// Finalize the outer cells of diagonal d (Np <= 64, cell images; one CTA per cell):
// adds the candidates that do not come from R0/R3/R4 and runs the inner wavefront of R1/R2/SW2.
//   base  i1==j1 && i2==j2: inter(s1[i1], s2r[i2])            (assignment, eval_FTable :576)
//   S1(i1,j1)+S2(i2,j2)
//   SW2 = F(i1,j1,i2+1,j2-1)+intra(s2r[i2],s2r[j2]) if j2-i2>=4
//   R1 (:614-640) max_{k2} F(i1,j1,i2,k2)+S2(k2+1,j2); R2 (:641-667) max_{k2} S2(i2,k2)+F(i1,j1,k2+1,j2)
// F arrives holding max(R0,R3,R4,SW1) (or +0): SW1 = F(i1+1,j1-1,.)+intra(s1[i1],s1[j1])
// (V3/bpmax_outer_south_west.c:115-160) was stored into this cell's still-cleared table by the
// finalize of (i1+1, j1-1) two diagonals earlier, before any product touched it. Every literal-0
// candidate is covered because every value is >= +0. Writes the cell's blocks (-inf outside the
// logical triangle, S1(i1,j1) on the subdiagonal) and its S1 pieces.
// The inner wavefront pushes forward: every inner cell (i2,j2), e2 = j2-i2 >= 1, has one owner
// thread that keeps its running maximum in a register. When inner diagonal e is final, each
// owner adds its two candidates that read diagonal e,
//   R1 with k2 = i2+e:    F[i2][i2+e] + S2(i2+e+1, j2)
//   R2 with k2 = j2-e-1:  S2(i2, j2-e-1) + F[j2-e][j2]
// to every open cell (e2 > e); the cells of diagonal e+1 have then seen all their R1/R2 terms
// and are final after SW2. One CTA barrier per inner diagonal; the diagonals are kept in shared
// memory diagonal-major, D[e][i2] = F[i2][i2+e].
// CTAs after the first njobs compute S1 on diagonal d+1 (V3/bpmax_verify.c:533-544), one warp
// per cell, from S1 diagonals <= d (S1 is cleared to 0 before the fill; j-i <= 3 stays 0).
// ------------------------------------------------------------------------------------------
struct CellJob {
    int pair, i1;
};

// threads per cell: the wavefront's serial work per step is K owned cells per thread. Fewer
// threads per cell cost latency per cell but issue fewer instructions per step in total, which pays
// when a launch holds many more cells than the GPU runs at once (FIN_WIDE_CELLS below)
constexpr int fin_threads(int NP) { return NP >= 48 ? 512 : (NP >= 24 ? 256 : 64); }
// element (r, c) of tile (I2, J2) of an outer cell in the reference layout (tiles of T+1 rows, the
// last one the halo; R = padding rows/columns of the first tile row/column); val(i2, j2) gives the
// cell's inner value for 0 <= i2 <= j2 < N, the only entries read
template <class Val>
__device__ __forceinline__ float reference_tile_elem_v(const Val &val, int T, int R, int I2, int J2, int r, int c)
{
    const int Ri = I2 == 0 ? R : 0, Rj = (I2 == 0 && J2 == 0) ? R : 0;
    float v = __int_as_float(0x7fc00000);  // NaN: a cell the reference leaves unwritten
    if (I2 <= J2 && c >= Rj) {
        if (r < T) {
            if (r >= Ri) {
                const int i2 = I2 * T + r - R, j2 = J2 * T + c - R;
                v = i2 <= j2 ? val(i2, j2) : -3.402823466e+38f;
            }
        } else {
            v = I2 == J2 ? -3.402823466e+38f : val((I2 + 1) * T - R, J2 * T + c - R);
        }
    }
    return v;
}
__device__ __forceinline__ float reference_tile_elem(const PairDesc &pd, const float *__restrict__ F, long long cell,
                                                     int T, int R, int I2, int J2, int r, int c)
{
    return reference_tile_elem_v([&](int i2, int j2) { return f_value(pd, F, cell, i2, j2); }, T, R, I2, J2, r, c);
}

// element `rem` (in [0, Ns*Ns*(T+1)*T)) of outer cell (i1, j1) in the reference layout
__device__ __forceinline__ float reference_elem(const PairDesc &pd, const float *__restrict__ F, int T, int Ns, int R,
                                                int i1, int j1, long long rem)
{
    const long long tile_f = (long long)(T + 1) * T;
    const int I2 = (int)(rem / ((long long)Ns * tile_f));
    rem %= (long long)Ns * tile_f;
    const int J2 = (int)(rem / tile_f);
    rem %= tile_f;
    return reference_tile_elem(pd, F, cell_index(pd.M, i1, j1), T, R, I2, J2, (int)(rem / T), (int)(rem % T));
}

// Reference-layout copy of the cells a finalize launch completes (the copy-out of bpmax_gpu_fill):
// out == nullptr for none; else cell (i1, i1+d) of the (single) pair goes to
// out + (d*M - d(d-1)/2 + i1) * cell_f, diagonal after diagonal, in the reference's tile layout of
// N_tile = T (Ns tiles a side; see reference_elem)
struct RefOut {
    float *out;
    int T, Ns;
};

constexpr int FIN_BULK_THREADS = 256;  // widths >= 48, launches of FIN_BULK_CELLS cells or more
constexpr int FIN_BULK_CELLS = 2048;

template <int NP, int T = fin_threads(NP)>
struct FinShape {
    static constexpr int THREADS = T;
    static constexpr int WARPS = THREADS / 32;
    static constexpr int K = (NP * (NP - 1) / 2 + THREADS - 1) / THREADS;  // owned inner cells per thread
    static constexpr int MINB = 1536 / THREADS;  // 48 resident warps per SM (at most 40 registers)
    static_assert(K <= 8, "the step switch covers 8 slots");
    static constexpr size_t SMEM = 2 * (size_t)NP * NP * sizeof(float) + NP;  // D, S2, bases
};

// first float of row e of a triangular diagonal-major table of width NP (row e holds NP - e entries)
__host__ __device__ __forceinline__ int drow(int NP, int e) { return e * NP - e * (e - 1) / 2; }

// (BI, BJ) of the q-th block of the upper block triangle (row-major triangle order)
__device__ __forceinline__ void blk_decode(int NB, int q, int &BI, int &BJ)
{
    BI = 0;
    while (q >= NB - BI) { q -= NB - BI; ++BI; }
    BJ = BI + q;
}

template <int NP, int T = fin_threads(NP)>
__global__ void __launch_bounds__(FinShape<NP, T>::THREADS, FinShape<NP, T>::MINB)
finalize_small_kernel(const CellJob *__restrict__ jobs, int njobs, const CellJob *__restrict__ s1jobs, int ns1,
                      const PairDesc *__restrict__ pairs, float *__restrict__ F, float *__restrict__ S,
                      const uint8_t *__restrict__ bases, Weights W, int d, RefOut ro)
{
    using Sh = FinShape<NP, T>;
    constexpr int NB = NP / 8, NBLK = NB * (NB + 1) / 2, K = Sh::K;
    constexpr long long CELL = 4LL * R0_TAB_COLBASE[NB][NB];
    extern __shared__ __align__(16) float fsm[];
    float *D = fsm, *S2s = fsm + NP * NP;
    uint8_t *sb = reinterpret_cast<uint8_t *>(fsm + 2 * NP * NP);
    __shared__ int cbs[NB];    // float offset of each block column in the cell image
    __shared__ float wsh[12];  // the weight table (indexed by pair type)
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid < 12) wsh[tid] = W.w[tid];
    if (tid < NB) cbs[tid] = 4 * c_img_colbase[NB][tid];
    __syncthreads();
    if ((int)blockIdx.x >= njobs) {  // S1 cells (i, i+d+1), one per warp
        const int q = ((int)blockIdx.x - njobs) * Sh::WARPS + warp;
        if (q >= ns1) return;
        const CellJob job = s1jobs[q];
        const PairDesc pd = pairs[job.pair];
        const int M = pd.M, i = job.i1, j = i + d + 1;
        float *S1 = S + pd.S1_off;
        if (j - i <= 3) return;  // stays 0
        const uint8_t *s1 = bases + pd.seq1_off;
        float r0 = NEG_INF, r1 = NEG_INF;
        int k = i + lane;
        for (; k + 32 < j; k += 64) {
            r0 = fmaxf(r0, S1[i * M + k] + S1[(k + 1) * M + j]);
            r1 = fmaxf(r1, S1[i * M + k + 32] + S1[(k + 33) * M + j]);
        }
        if (k < j) r0 = fmaxf(r0, S1[i * M + k] + S1[(k + 1) * M + j]);
        float red = fmaxf(r0, r1);
        for (int o = 16; o > 0; o >>= 1) red = fmaxf(red, __shfl_xor_sync(0xffffffffu, red, o));
        if (lane == 0) S1[i * M + j] = fmaxf(S1[(i + 1) * M + (j - 1)] + score_w(wsh, s1[i], s1[j]), red);
        return;
    }
    const CellJob job = jobs[blockIdx.x];
    const PairDesc pd = pairs[job.pair];
    const int M = pd.M, N = pd.N, i1 = job.i1, j1 = i1 + d;
    float *Fc = F + pd.F_off + cell_index(M, i1, j1) * CELL;
    const float *S1 = S + pd.S1_off;
    const float *S2 = S + pd.S2_off;
    const uint8_t *s1 = bases + pd.seq1_off;
    const uint8_t *s2r = bases + pd.seq2_off;
    const float s1v = S1[i1 * M + j1];
    for (int q4 = tid; q4 < NP * NP / 4; q4 += Sh::THREADS)
        *reinterpret_cast<float4 *>(S2s + 4 * q4) = *reinterpret_cast<const float4 *>(S2 + 4 * q4);
    for (int q = tid; q < NP; q += Sh::THREADS) sb[q] = q < N ? s2r[q] : 4;
    __syncthreads();
    // accumulated value of inner cell (r, c), r <= c, from the cell image
    auto img = [&](int r, int c) { return Fc[cbs[c >> 3] + 68 * (r >> 3) + 8 * (r & 7) + (c & 7)]; };
    // owned inner cells c = tid + THREADS*k among the N(N-1)/2 cells with e2 >= 1, ordered by
    // (e2, i2): running maxima start at max(accumulated, S1+S2)
    const int ncells = N * (N - 1) / 2;
    int cell_i[K], cell_e[K];
    float acc[K], sw2[K];  // running maximum; SW2 weight (-inf: no SW2 term)
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const int c = tid + Sh::THREADS * k;
        cell_e[k] = NP;  // no cell: never open
        cell_i[k] = 0;
        acc[k] = NEG_INF;
        sw2[k] = NEG_INF;
        if (c < ncells) {
            int e = 1, rem = c;
            while (rem >= N - e) { rem -= N - e; ++e; }
            cell_e[k] = e;
            cell_i[k] = rem;
            acc[k] = fmaxf(img(rem, rem + e), s1v + S2s[rem * NP + rem + e]);
            if (e >= 4) sw2[k] = score_w(wsh, sb[rem], sb[rem + e]);
        }
    }
    if (tid < N)  // inner diagonal 0
        D[tid] = d == 0 ? score_w(wsh + 6, s1[i1], sb[tid]) : fmaxf(img(tid, tid), s1v + S2s[tid * NP + tid]);
    __syncthreads();
    // slot k of every thread holds cells THREADS*k .. THREADS*(k+1)-1 of the (e2, i2) order, so the
    // slots whose cells are all final (e2 <= e) are the same for every thread: the step enters the
    // unrolled slot sequence at the first slot still open (a CTA-uniform branch), instead of
    // evaluating the closed slots under a false predicate
    auto step = [&](auto kc, int e, const float *De) {
        constexpr int k = decltype(kc)::value;
        if constexpr (k < K) {
            const int e2 = cell_e[k];
            if (e2 > e && e2 < NP) {
                const int i2 = cell_i[k], j2 = i2 + e2;
                acc[k] = fmax3(acc[k], De[i2] + S2s[(i2 + e + 1) * NP + j2], S2s[i2 * NP + j2 - e - 1] + De[j2 - e]);
                if (e2 == e + 1)  // all R1/R2 terms seen: SW2, then the cell is final
                    D[e2 * NP + i2] = fmaxf(acc[k], D[max(e2 - 2, 0) * NP + i2 + 1] + sw2[k]);
            }
        }
    };
    for (int e = 0; e + 1 < N; ++e) {
        const float *De = D + e * NP;
        const int first = (e * N - e * (e + 1) / 2) / Sh::THREADS;  // cells with e2 <= e come first
        switch (first) {
        case 0: step(std::integral_constant<int, 0>{}, e, De); [[fallthrough]];
        case 1: step(std::integral_constant<int, 1>{}, e, De); [[fallthrough]];
        case 2: step(std::integral_constant<int, 2>{}, e, De); [[fallthrough]];
        case 3: step(std::integral_constant<int, 3>{}, e, De); [[fallthrough]];
        case 4: step(std::integral_constant<int, 4>{}, e, De); [[fallthrough]];
        case 5: step(std::integral_constant<int, 5>{}, e, De); [[fallthrough]];
        case 6: step(std::integral_constant<int, 6>{}, e, De); [[fallthrough]];
        case 7: step(std::integral_constant<int, 7>{}, e, De); [[fallthrough]];
        default: break;
        }
        __syncthreads();
    }
    // write-back, 4 columns of one block row per step; SW1 candidate of cell (i1-1, j1+1), whose
    // table nothing else has written yet
    const bool push = i1 >= 1 && j1 + 1 < M && d + 2 >= 4;
    const float wp = push ? score_w(wsh, s1[i1 - 1], s1[j1 + 1]) : 0.0f;
    float *Fn = push ? F + pd.F_off + cell_index(M, i1 - 1, j1 + 1) * CELL : nullptr;
    for (int q4 = tid; q4 < NBLK * 16; q4 += Sh::THREADS) {
        int BI, BJ;
        blk_decode(NB, q4 >> 4, BI, BJ);
        const int r = 8 * BI + ((q4 & 15) >> 1), c0 = 8 * BJ + 4 * (q4 & 1);
        float v[4], u[4];
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            const int c = c0 + t;
            const bool valid = r <= c && c < N;
            v[t] = valid ? D[(c - r) * NP + r] : (r == c + 1 ? s1v : NEG_INF);  // S1 on the subdiagonal
            u[t] = valid ? v[t] + wp : 0.0f;
        }
        const int o = cbs[BJ] + 68 * BI + 4 * (q4 & 15);  // block (BI, BJ), row r & 7, half
        if (push) *reinterpret_cast<float4 *>(Fn + o) = make_float4(u[0], u[1], u[2], u[3]);
        *reinterpret_cast<float4 *>(Fc + o) = make_float4(v[0], v[1], v[2], v[3]);
    }
    if (tid < 2 * NB) {  // S1 piece of every block column: -inf x7, S1(i1,j1)
        const int BJ = tid >> 1, h = tid & 1;
        float4 p = make_float4(NEG_INF, NEG_INF, NEG_INF, NEG_INF);
        if (h == 1) p.w = s1v;
        *reinterpret_cast<float4 *>(Fc + cbs[BJ] + 68 * (BJ + 1) + 4 * h) = p;
    }
    if (ro.out) {  // this cell in the reference layout, from the final table in shared memory (the
                   // values the image holds), one warp per tile row of T floats
        const int TT = ro.T, R = (TT - N % TT) % TT, tile_rows = TT + 1, rows = ro.Ns * ro.Ns * tile_rows;
        float *dst = ro.out + ((long long)d * M - (long long)d * (d - 1) / 2 + i1) * ((long long)rows * TT);
        auto dval = [&](int i2, int j2) { return D[(j2 - i2) * NP + i2]; };
        for (int rr = warp; rr < rows; rr += Sh::WARPS) {
            const int I2 = rr / (ro.Ns * tile_rows), rem = rr % (ro.Ns * tile_rows);
            const int J2 = rem / tile_rows, r = rem % tile_rows;
            for (int c = lane; c < TT; c += 32) dst[rr * TT + c] = reference_tile_elem_v(dval, TT, R, I2, J2, r, c);
        }
    }
}

// ------------------------------------------------------------------------------------------
// Layout conversion: compact device tables -> the reference's linear layout for outer row i1
// (cells (i1, j1) for j1 in [i1, M)): out[(j1-i1)][I2][J2][r][c] of N_tile x (N_tile+1) tiles
// (V3/bpmax-wrapper.c:44, :175-197). Written cells follow V3/bpmax_ftable_init.c:171-214
// (-FLT_MAX masks, halo of diagonal tiles) and V3/bpmax_inner_reductions_finalize.c:132 (halo of
// off-diagonal tiles = row 0 of the tile below); cells the reference never writes become NaN.
// ------------------------------------------------------------------------------------------
__global__ void to_reference_row_kernel(const PairDesc *__restrict__ pdp, const float *__restrict__ F, int T, int Ns,
                                        int i1, long long n_out, float *__restrict__ out)
{
    const PairDesc pd = *pdp;
    const int R = (T - pd.N % T) % T;
    const long long cell_f = (long long)Ns * Ns * (T + 1) * T;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n_out;
         q += (long long)gridDim.x * blockDim.x)
        out[q] = reference_elem(pd, F, T, Ns, R, i1, i1 + (int)(q / cell_f), q % cell_f);
}

// the same conversion for the cells of outer diagonal d (cells (i1, i1+d), i1 = 0 .. M-1-d), one
// after another in `out`: final all at once when the diagonal is, unlike a row
__global__ void to_reference_diag_kernel(const PairDesc *__restrict__ pdp, const float *__restrict__ F, int T, int Ns,
                                         int d, long long n_out, float *__restrict__ out)
{
    const PairDesc pd = *pdp;
    const int R = (T - pd.N % T) % T;
    const long long cell_f = (long long)Ns * Ns * (T + 1) * T;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n_out;
         q += (long long)gridDim.x * blockDim.x) {
        const int i1 = (int)(q / cell_f);
        out[q] = reference_elem(pd, F, T, Ns, R, i1, i1 + d, q % cell_f);
    }
}

// compact device tables -> dense compact host layout (stride N), -FLT_MAX below the diagonal
__global__ void to_compact_kernel(const PairDesc *__restrict__ pdp, const float *__restrict__ F, long long n_out,
                                  float *__restrict__ out)
{
    const PairDesc pd = *pdp;
    const int N = pd.N;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n_out;
         q += (long long)gridDim.x * blockDim.x) {
        const long long c = q / ((long long)N * N);
        const int r = (int)((q / N) % N), col = (int)(q % N);
        out[q] = r <= col ? f_value(pd, F, c, r, col) : -3.402823466e+38f;
    }
}

// inner tables of the outer cells (i1, j1), i1 in [i1_lo, i1_lo+nI), j1 in [j1_lo, j1_lo+nJ), of one
// pair -> out[i1-i1_lo][j1-j1_lo][N][N]; -FLT_MAX where i2 > j2, NaN for outer cells with i1 > j1
__global__ void read_cells_kernel(const PairDesc *__restrict__ pdp, const float *__restrict__ F, int i1_lo, int j1_lo,
                                  int nJ, long long n_out, float *__restrict__ out)
{
    const PairDesc pd = *pdp;
    const long long NN = (long long)pd.N * pd.N;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n_out;
         q += (long long)gridDim.x * blockDim.x) {
        const long long oc = q / NN;
        const int i1 = i1_lo + (int)(oc / nJ), j1 = j1_lo + (int)(oc % nJ);
        const int r = (int)((q % NN) / pd.N), c = (int)(q % pd.N);
        float v = __int_as_float(0x7fc00000);
        if (i1 <= j1) v = r <= c ? f_value(pd, F, cell_index(pd.M, i1, j1), r, c) : -3.402823466e+38f;
        out[q] = v;
    }
}

__global__ void gather_scores_kernel(const PairDesc *__restrict__ pairs, const float *__restrict__ F, int num_pairs,
                                     float *__restrict__ scores)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= num_pairs) return;
    const PairDesc pd = pairs[p];
    scores[p] = f_value(pd, F, cell_index(pd.M, 0, pd.M - 1), 0, pd.N - 1);
}

// ------------------------------------------------------------------------------------------
// Max-plus issue ceiling: the product kernel's instruction mix with nothing to share between
// candidates. Each step of a chain is one packed add (two candidate sums, the running operand
// plus a step) and one 3-input max that merges both sums into the chain's maximum; every sum is
// new (the running operand changes each step) and is consumed once, so the compiler can neither
// hoist nor reuse an add. MAXPLUS_PEAK_CHAINS independent chains per thread give the schedulers
// the same independent work as the product kernel's 8x8 tile. Each iteration is
// 4 * 2 * MAXPLUS_PEAK_CHAINS candidates per thread.
// ------------------------------------------------------------------------------------------
constexpr int MAXPLUS_PEAK_CHAINS = 16;
__global__ void __launch_bounds__(128) maxplus_peak_kernel(const float *__restrict__ in, float *__restrict__ out,
                                                           int reps)
{
    constexpr int CH = MAXPLUS_PEAK_CHAINS;
    float2 p[CH], q[CH];
    float m[CH];
#pragma unroll
    for (int i = 0; i < CH; ++i) {
        p[i] = make_float2(in[(threadIdx.x + i) & 63], in[(threadIdx.x + 2 * i + 1) & 63]);
        q[i] = make_float2(in[(threadIdx.x + 3 * i + 2) & 63] * 1e-7f, in[(threadIdx.x + 5 * i + 3) & 63] * 1e-7f);
        m[i] = NEG_INF;
    }
    for (int r = 0; r < reps; ++r) {
#pragma unroll
        for (int s = 0; s < 4; ++s)
#pragma unroll
            for (int i = 0; i < CH; ++i) {
                p[i] = __fadd2_rn(p[i], q[i]);
                m[i] = fmax3(m[i], p[i].x, p[i].y);
            }
    }
    float s = 0.f;
#pragma unroll
    for (int i = 0; i < CH; ++i) s += p[i].x + p[i].y + m[i];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace bpmax
