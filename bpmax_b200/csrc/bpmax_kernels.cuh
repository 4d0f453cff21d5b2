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
//   F [c][Np][Np]  row-major inner table, i2 over the reversed strand 2, -inf where i2>j2 or
//                  i2,j2 >= N (Np = N rounded up to a multiple of 8)
//   FT[c][Np][Np]  the same table transposed, written once per cell, so the A operand of the
//                  max-plus product streams into shared memory with plain 16-byte copies
//   S1[M][M], S2[Np][Np] single-strand tables (S2 over the reversed strand 2)
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace bpmax {

constexpr float NEG_INF = -__builtin_inff();

struct Weights {
    float w[12];  // intra AU,UA,GC,CG,GU,UG ; inter AU,UA,GC,CG,GU,UG
};

struct PairDesc {
    int M, N, Np, pad0;
    long long F_off;   // float offset of F[0] (and of FT[0] in the FT arena)
    long long S1_off;  // float offset of S1 in the S arena
    long long S2_off;  // float offset of S2 in the S arena
    int seq1_off;      // offset of seq1 in the base arena (uint8)
    int seq2_off;      // offset of the REVERSED seq2 in the base arena (uint8)
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
// Single-strand table (V3/bpmax_verify.c:533-544 for S1, :560-571 for S2 over the reversed
// strand): S(i,j) = 0 if j-i<=3, else max(S(i+1,j-1)+intra(s[i],s[j]), max_{i<=k<j} S(i,k)+S(k+1,j)).
// One CTA per (pair, strand); wavefront over the diagonal j-i. Cells of S2 outside the N x N
// upper triangle are left at 0 and never read.
// ------------------------------------------------------------------------------------------
__global__ void single_strand_kernel(const PairDesc *__restrict__ pairs, const uint8_t *__restrict__ bases,
                                     float *__restrict__ S, Weights W)
{
    const PairDesc pd = pairs[blockIdx.x >> 1];
    const bool second = blockIdx.x & 1;
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
// R0 + R3 + R4 for inner tables of width Np = 8*NB <= 64 (one CTA per job: one outer cell and
// a range of k1).
//   R0 (V3/bpmax_verify.c:584-613):  max_{k1,k2} F(i1,k1,i2,k2) + F(k1+1,j1,k2+1,j2)
//   R3 (:668-694):                    max_{k1}   S1(i1,k1) + F(k1+1,j1,i2,j2)
//   R4 (:695-721):                    max_{k1}   F(i1,k1,i2,j2) + S1(k1+1,j1)
// For one k1, R0 is a product of two upper-triangular matrices in the (max,+) semiring:
//   C[i2][j2] = max_{k2} A[i2][k2] + B'[k2][j2],  A = F(i1,k1), B'[k2] = row k2+1 of F(k1+1,j1).
// Shared memory holds A^T (from the FT copy) and B, both padded to a row stride of Np+4 floats.
// The triangular product is split into tasks (bi,bj,kb): an 8x8 output micro-tile (bi,bj)
// times one 8-wide k2 block kb, bi<=kb<=bj; every task is 8 k-steps of a 8x8 register tile,
// so all threads do the same work. Tasks of one micro-tile live in different threads; their
// partial maxima, like those of the CTAs that share the cell, merge by atomicMax into F.
// ------------------------------------------------------------------------------------------
struct R0Job {
    int pair, i1, k1a, k1b;  // cell (i1, i1+d) of pair, k1 in [k1a, k1b)
};

template <int NB>
struct R0Shape {
    static constexpr int NP = 8 * NB;
    static constexpr int LD = NP + 4;                 // smem row stride (floats)
    static constexpr int A_FLOATS = NP * LD;          // A^T[k2][i2]
    static constexpr int B_FLOATS = (NP + 1) * LD;    // B[r][j2], r = 0..NP (row NP = -inf)
    static constexpr int STAGE = A_FLOATS + B_FLOATS;
    static constexpr int TASKS = NB * (NB + 1) * (NB + 2) / 6;
    static constexpr int THREADS = 128;
    static constexpr int NSEG = (NP + 31) / 32;        // R3/R4 row segments per row
    static constexpr int SEGW = NP / NSEG;             // segment width (a multiple of 4)
    static constexpr int R34_THREADS = NP * NSEG;
    static constexpr size_t SMEM = 2 * (size_t)STAGE * sizeof(float);
};

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

template <int NB>
__global__ void __launch_bounds__(128, 2)
r0_small_kernel(const R0Job *__restrict__ jobs, const PairDesc *__restrict__ pairs, float *__restrict__ F,
                const float *__restrict__ FT, const float *__restrict__ S, int d)
{
    using Sh = R0Shape<NB>;
    constexpr int NP = Sh::NP, LD = Sh::LD;
    extern __shared__ __align__(16) float smem[];
    const R0Job job = jobs[blockIdx.x];
    const PairDesc pd = pairs[job.pair];
    const int M = pd.M, N = pd.N, i1 = job.i1, j1 = i1 + d;
    const float *S1 = S + pd.S1_off;
    const long long tile = (long long)NP * NP;
    const float *Fp = F + pd.F_off;
    const float *FTp = FT + pd.F_off;
    const int tid = threadIdx.x;

    // row NP of B in both stages is -inf (B'[NP-1] beyond the table); never overwritten
    for (int c = tid; c < LD; c += Sh::THREADS) {
        smem[Sh::A_FLOATS + NP * LD + c] = NEG_INF;
        smem[Sh::STAGE + Sh::A_FLOATS + NP * LD + c] = NEG_INF;
    }

    auto load_stage = [&](int stage, int k1) {
        float *As = smem + stage * Sh::STAGE;
        float *Bs = As + Sh::A_FLOATS;
        const float *ga = FTp + cell_index(M, i1, k1) * tile;      // A^T = FT(i1,k1)
        const float *gb = Fp + cell_index(M, k1 + 1, j1) * tile;   // B   = F(k1+1,j1)
        constexpr int CPR = NP / 4;                                 // 16-byte chunks per row
        for (int q = tid; q < 2 * NP * CPR; q += Sh::THREADS) {
            const int which = q / (NP * CPR), rr = (q / CPR) % NP, cc = (q % CPR) * 4;
            if (which == 0) cp_async16(As + rr * LD + cc, ga + rr * NP + cc);
            else cp_async16(Bs + rr * LD + cc, gb + rr * NP + cc);
        }
        cp_async_commit();
    };

    // task of this thread: micro-tile (bi,bj), k-block kb
    int bi = 0, bj = 0, kb = 0;
    const bool has_task = tid < Sh::TASKS;
    {
        int t = tid, found = 0;
        for (int a = 0; a < NB && !found; ++a)
            for (int b = a; b < NB && !found; ++b) {
                const int n = b - a + 1;
                if (t < n) { bi = a; bj = b; kb = a + t; found = 1; }
                else t -= n;
            }
    }
    // R3/R4 ownership: row r of B (R3 cells (r, c..c+SEGW)), row r of A^T (R4 cells (c.., r))
    const bool has34 = tid < Sh::R34_THREADS;
    const int r34 = tid / Sh::NSEG, c34 = (tid % Sh::NSEG) * Sh::SEGW;

    float acc[8][8];
    float acc3[Sh::SEGW], acc4[Sh::SEGW];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = NEG_INF;
#pragma unroll
    for (int i = 0; i < Sh::SEGW; ++i) { acc3[i] = NEG_INF; acc4[i] = NEG_INF; }

    load_stage(0, job.k1a);
    for (int k1 = job.k1a; k1 < job.k1b; ++k1) {
        const int stage = (k1 - job.k1a) & 1;
        if (k1 + 1 < job.k1b) { load_stage(stage ^ 1, k1 + 1); cp_async_wait<1>(); }
        else cp_async_wait<0>();
        __syncthreads();
        const float *As = smem + stage * Sh::STAGE;
        const float *Bs = As + Sh::A_FLOATS;
        if (has_task) {
            const float *pa = As + (8 * kb) * LD + 8 * bi;
            const float *pb = Bs + (8 * kb + 1) * LD + 8 * bj;
#pragma unroll
            for (int k = 0; k < 8; k += 2) {
                const float4 a0 = *reinterpret_cast<const float4 *>(pa + k * LD);
                const float4 a1 = *reinterpret_cast<const float4 *>(pa + k * LD + 4);
                const float4 a2 = *reinterpret_cast<const float4 *>(pa + (k + 1) * LD);
                const float4 a3 = *reinterpret_cast<const float4 *>(pa + (k + 1) * LD + 4);
                const float4 b0 = *reinterpret_cast<const float4 *>(pb + k * LD);
                const float4 b1 = *reinterpret_cast<const float4 *>(pb + k * LD + 4);
                const float4 b2 = *reinterpret_cast<const float4 *>(pb + (k + 1) * LD);
                const float4 b3 = *reinterpret_cast<const float4 *>(pb + (k + 1) * LD + 4);
                const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
                const float aw[8] = {a2.x, a2.y, a2.z, a2.w, a3.x, a3.y, a3.z, a3.w};
                const float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
                const float bw[8] = {b2.x, b2.y, b2.z, b2.w, b3.x, b3.y, b3.z, b3.w};
#pragma unroll
                for (int i = 0; i < 8; ++i)
#pragma unroll
                    for (int j = 0; j < 8; ++j) acc[i][j] = fmax3(acc[i][j], av[i] + bv[j], aw[i] + bw[j]);
            }
        }
        if (has34) {
            const float s1a = S1[i1 * M + k1], s1b = S1[(k1 + 1) * M + j1];
            const float *rb = Bs + r34 * LD + c34;  // F(k1+1,j1)[r34][c34 + x]
            const float *ra = As + r34 * LD + c34;  // F(i1,k1)[c34 + x][r34]
#pragma unroll
            for (int x = 0; x < Sh::SEGW; x += 4) {
                const float4 vb = *reinterpret_cast<const float4 *>(rb + x);
                const float4 va = *reinterpret_cast<const float4 *>(ra + x);
                acc3[x + 0] = fmaxf(acc3[x + 0], s1a + vb.x);
                acc3[x + 1] = fmaxf(acc3[x + 1], s1a + vb.y);
                acc3[x + 2] = fmaxf(acc3[x + 2], s1a + vb.z);
                acc3[x + 3] = fmaxf(acc3[x + 3], s1a + vb.w);
                acc4[x + 0] = fmaxf(acc4[x + 0], va.x + s1b);
                acc4[x + 1] = fmaxf(acc4[x + 1], va.y + s1b);
                acc4[x + 2] = fmaxf(acc4[x + 2], va.z + s1b);
                acc4[x + 3] = fmaxf(acc4[x + 3], va.w + s1b);
            }
        }
        __syncthreads();
    }

    int *out = reinterpret_cast<int *>(F + pd.F_off + cell_index(M, i1, j1) * tile);
    if (has_task) {
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int i2 = 8 * bi + i, j2 = 8 * bj + j;
                if (i2 < j2 && j2 < N) atomicMax(out + i2 * NP + j2, __float_as_int(acc[i][j]));
            }
    }
    if (has34) {
#pragma unroll
        for (int x = 0; x < Sh::SEGW; ++x) {
            const int c = c34 + x;
            if (r34 <= c && c < N) atomicMax(out + r34 * NP + c, __float_as_int(acc3[x]));  // R3 at (r34, c)
            if (c <= r34 && r34 < N) atomicMax(out + c * NP + r34, __float_as_int(acc4[x]));  // R4 at (c, r34)
        }
    }
}

// ------------------------------------------------------------------------------------------
// Finalize one outer cell (one CTA per cell of diagonal d, Np <= 64): adds the candidates that
// do not come from R0/R3/R4 and runs the inner wavefront of R1/R2/SW2 in shared memory.
//   base  i1==j1 && i2==j2: inter(s1[i1], s2r[i2])            (assignment, eval_FTable :576)
//   S1(i1,j1)+S2(i2,j2); SW1 = F(i1+1,j1-1,i2,j2)+intra(s1[i1],s1[j1]) if j1-i1>=4
//   SW2 = F(i1,j1,i2+1,j2-1)+intra(s2r[i2],s2r[j2]) if j2-i2>=4
//   R1 (:614-640) max_{k2} F(i1,j1,i2,k2)+S2(k2+1,j2); R2 (:641-667) max_{k2} S2(i2,k2)+F(i1,j1,k2+1,j2)
// F arrives holding max(R0,R3,R4) (or 0 on a cleared cell); all literal-0 candidates are
// covered because every value is >= +0. Writes F and FT, -inf outside the logical triangle.
// ------------------------------------------------------------------------------------------
struct CellJob {
    int pair, i1;
};

template <int NP>
__global__ void __launch_bounds__(256)
finalize_small_kernel(const CellJob *__restrict__ jobs, const PairDesc *__restrict__ pairs,
                      float *__restrict__ F, float *__restrict__ FT, const float *__restrict__ S,
                      const uint8_t *__restrict__ bases, Weights W, int d)
{
    constexpr int LD = NP + 1;
    __shared__ float Fs[NP * LD];
    __shared__ float Ss[(NP + 1) * LD];
    __shared__ uint8_t sb[NP];
    const CellJob job = jobs[blockIdx.x];
    const PairDesc pd = pairs[job.pair];
    const int M = pd.M, N = pd.N, i1 = job.i1, j1 = i1 + d;
    const long long tile = (long long)NP * NP;
    float *Fc = F + pd.F_off + cell_index(M, i1, j1) * tile;
    float *FTc = FT + pd.F_off + cell_index(M, i1, j1) * tile;
    const float *S1 = S + pd.S1_off;
    const float *S2 = S + pd.S2_off;
    const uint8_t *s1 = bases + pd.seq1_off;
    const uint8_t *s2r = bases + pd.seq2_off;
    const int tid = threadIdx.x, nt = blockDim.x;
    const float s1v = S1[i1 * M + j1];
    const bool sw1 = d >= 4;
    const float w1 = sw1 ? score_w(W.w, s1[i1], s1[j1]) : 0.0f;
    const float *Fsw = sw1 ? F + pd.F_off + cell_index(M, i1 + 1, j1 - 1) * tile : nullptr;

    for (int q = tid; q < NP; q += nt) sb[q] = q < N ? s2r[q] : 4;
    for (int q = tid; q < (NP + 1) * LD; q += nt) {
        const int r = q / LD, c = q % LD;
        Ss[q] = (r < N && c < N) ? S2[r * NP + c] : 0.0f;
    }
    for (int q = tid; q < NP * NP; q += nt) {
        const int r = q / NP, c = q % NP;
        float v = NEG_INF;
        if (r <= c && c < N) {
            if (d == 0 && r == c) {
                v = score_w(W.w + 6, s1[i1], s2r[r]);
            } else {
                v = fmaxf(Fc[q], s1v + S2[r * NP + c]);
                if (sw1) v = fmaxf(v, Fsw[q] + w1);
            }
        }
        Fs[r * LD + c] = v;
    }
    __syncthreads();
    for (int dd = 1; dd < N; ++dd) {
        const int cells = N - dd;
        int g = 1;
        while (g < 32 && g * 2 * cells <= nt) g *= 2;
        const int lane_g = tid & (g - 1);
        const int slots = nt / g;
        for (int base = 0; base < cells; base += slots) {
            const int i2 = base + tid / g, j2 = i2 + dd;
            const bool act = i2 < cells;
            float red = NEG_INF;
            if (act)
                for (int k = i2 + lane_g; k < j2; k += g)
                    red = fmax3(red, Fs[i2 * LD + k] + Ss[(k + 1) * LD + j2], Ss[i2 * LD + k] + Fs[(k + 1) * LD + j2]);
            for (int o = g >> 1; o > 0; o >>= 1) red = fmaxf(red, __shfl_xor_sync(0xffffffffu, red, o, g));
            if (act && lane_g == 0) {
                float v = fmaxf(Fs[i2 * LD + j2], red);
                if (dd >= 4) v = fmaxf(v, Fs[(i2 + 1) * LD + (j2 - 1)] + score_w(W.w, sb[i2], sb[j2]));
                Fs[i2 * LD + j2] = v;
            }
        }
        __syncthreads();
    }
    for (int q = tid; q < NP * NP; q += nt) {
        const int r = q / NP, c = q % NP;
        Fc[q] = Fs[r * LD + c];
        FTc[q] = Fs[c * LD + r];
    }
}

// ------------------------------------------------------------------------------------------
// Layout conversion: compact device tables -> the reference's linear layout for outer row i1
// (cells (i1, j1) for j1 in [i1, M)): out[(j1-i1)][I2][J2][r][c] of N_tile x (N_tile+1) tiles
// (V3/bpmax-wrapper.c:44, :175-197). Written cells follow V3/bpmax_ftable_init.c:171-214
// (-FLT_MAX masks, halo of diagonal tiles) and V3/bpmax_inner_reductions_finalize.c:132 (halo of
// off-diagonal tiles = row 0 of the tile below); cells the reference never writes become NaN.
// ------------------------------------------------------------------------------------------
__global__ void to_reference_row_kernel(const float *__restrict__ F, int M, int N, int Np, int T, int Ns,
                                        int i1, long long n_out, float *__restrict__ out)
{
    const int R = (T - N % T) % T;
    const long long tile_f = (long long)(T + 1) * T;
    const long long cell_f = (long long)Ns * Ns * tile_f;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n_out;
         q += (long long)gridDim.x * blockDim.x) {
        const int j1 = i1 + (int)(q / cell_f);
        long long rem = q % cell_f;
        const int I2 = (int)(rem / ((long long)Ns * tile_f));
        rem %= (long long)Ns * tile_f;
        const int J2 = (int)(rem / tile_f);
        rem %= tile_f;
        const int r = (int)(rem / T), c = (int)(rem % T);
        const float *C = F + cell_index(M, i1, j1) * (long long)Np * Np;
        const int Ri = I2 == 0 ? R : 0, Rj = (I2 == 0 && J2 == 0) ? R : 0;
        float v = __int_as_float(0x7fc00000);  // NaN: a cell the reference leaves unwritten
        if (I2 <= J2 && c >= Rj) {
            if (r < T) {
                if (r >= Ri) {
                    const int i2 = I2 * T + r - R, j2 = J2 * T + c - R;
                    v = i2 <= j2 ? C[(long long)i2 * Np + j2] : -3.402823466e+38f;
                }
            } else {
                v = I2 == J2 ? -3.402823466e+38f : C[(long long)((I2 + 1) * T - R) * Np + (J2 * T + c - R)];
            }
        }
        out[q] = v;
    }
}

// compact device tables (stride Np) -> dense compact host layout (stride N), -FLT_MAX below
__global__ void to_compact_kernel(const float *__restrict__ F, int M, int N, int Np, long long n_out,
                                  float *__restrict__ out)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n_out;
         q += (long long)gridDim.x * blockDim.x) {
        const long long c = q / ((long long)N * N);
        const int r = (int)((q / N) % N), col = (int)(q % N);
        out[q] = r <= col ? F[c * (long long)Np * Np + (long long)r * Np + col] : -3.402823466e+38f;
    }
}

__global__ void gather_scores_kernel(const PairDesc *__restrict__ pairs, const float *__restrict__ F, int num_pairs,
                                     float *__restrict__ scores)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= num_pairs) return;
    const PairDesc pd = pairs[p];
    scores[p] = F[pd.F_off + cell_index(pd.M, 0, pd.M - 1) * (long long)pd.Np * pd.Np + (pd.N - 1)];
}

// ------------------------------------------------------------------------------------------
// Max-plus issue ceiling: 8x8 register tile, two k-steps per 3-input max, operands perturbed
// once per iteration so nothing is loop-invariant. Each iteration is 128 candidates per thread.
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(128) maxplus_peak_kernel(const float *__restrict__ in, float *__restrict__ out,
                                                           int reps)
{
    float a[8], b[8], acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i) { a[i] = in[(threadIdx.x + i) & 63]; b[i] = in[(threadIdx.x + 8 + i) & 63]; }
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = NEG_INF;
    for (int r = 0; r < reps; ++r) {
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
            for (int j = 0; j < 8; ++j) acc[i][j] = fmax3(acc[i][j], a[i] + b[j], b[i] + a[j]);
#pragma unroll
        for (int i = 0; i < 8; ++i) { a[i] = a[i] * 0.999f; b[i] = b[i] * 1.001f; }
    }
    float s = 0.f;
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) s += acc[i][j];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace bpmax
