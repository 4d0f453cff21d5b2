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
    long long S2m_off; // Np > 64 only: S2 with -inf outside its triangle
    long long S2t_off; // Np > 64 only: ST1[j][k] = S2(k+1, j), -inf outside
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
// Single-strand table S2 over the reversed strand 2 (V3/bpmax_verify.c:560-571):
// S(i,j) = 0 if j-i<=3, else max(S(i+1,j-1)+intra(s[i],s[j]), max_{i<=k<j} S(i,k)+S(k+1,j)).
// One CTA per pair; wavefront over the diagonal j-i. Cells outside the N x N upper triangle are
// left at 0 and never read. (S1 is built diagonal by diagonal inside finalize_small_kernel.)
// ------------------------------------------------------------------------------------------
__global__ void single_strand_kernel(const PairDesc *__restrict__ pairs, const uint8_t *__restrict__ bases,
                                     float *__restrict__ S, Weights W)
{
    const PairDesc pd = pairs[blockIdx.x];
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
// R0 + R3 + R4 for inner tables of width Np = 8*NB <= 64 (one CTA per job: one outer cell and
// a range of k1).
//   R0 (V3/bpmax_verify.c:584-613):  max_{k1,k2} F(i1,k1,i2,k2) + F(k1+1,j1,k2+1,j2)
//   R3 (:668-694):                    max_{k1}   S1(i1,k1) + F(k1+1,j1,i2,j2)
//   R4 (:695-721):                    max_{k1}   F(i1,k1,i2,j2) + S1(k1+1,j1)
// Every finalized table F(a,b) stores S1(a,b) on its subdiagonal F[r][r-1] (never a logical
// cell). With A = F(i1,k1) shifted one column right, A_s[i2][k'] = A[i2][k'-1] (A_s[0][0] =
// S1(i1,k1)), and B = F(k1+1,j1) unshifted, one triangular (max,+) product gives all three:
//   max_{k' in [i2, j2+1]} A_s[i2][k'] + B[k'][j2]
//     k' = i2      : S1(i1,k1) + F(k1+1,j1)[i2][j2]                 (R3)
//     i2 < k' <= j2: F(i1,k1)[i2][k'-1] + F(k1+1,j1)[k'][j2]         (R0, k2 = k'-1)
//     k' = j2+1    : F(i1,k1)[i2][j2] + S1(k1+1,j1)                  (R4)
// and every other k' meets a -inf. Shared memory holds A_s k'-major (A_s^T[k'][i2], rows 1..Np
// copied from the FT table, row 0 = [S1(i1,k1), -inf...]) and B (rows 0..Np-1 of F, row Np =
// -inf except B[Np][Np-1] = S1(k1+1,j1)); 16-byte chunks that hold only masked entries are never
// copied (their shared slots stay -inf from the prologue), which halves the bytes per k1.
// The product is split into tasks (bi,bj,kb): 8x8 output micro-tile (bi,bj) times k' block
// [8kb, 8kb+8), bi<=kb<=bj, plus k' = 8bj+8 for the task with kb==bj. All tasks are 8 k-steps of
// an 8x8 register tile (fp32 add + 3-input max per two candidates). Tasks of one micro-tile live
// in different threads; their partial maxima, like those of the CTAs that share the cell, merge
// by atomicMax into F. For Np=64 the shared rows are unpadded and XOR-swizzled per 16-byte chunk
// and the task-to-lane table below makes every quarter-warp's 128-bit loads hit distinct banks.
// ------------------------------------------------------------------------------------------
struct R0Job {
    int pair, i1, k1a, k1b;  // cell (i1, i1+d) of pair, k1 in [k1a, k1b)
};

template <int NB>
struct R0Shape {
    static constexpr int NP = 8 * NB;
    static constexpr bool SWZ = NB == 8;              // swizzled, unpadded rows
    static constexpr int LD = SWZ ? NP : NP + 4;      // row stride (floats)
    static constexpr int CPR = NP / 4;                // 16-byte chunks per row
    static constexpr int ROWS = NP + 1;
    static constexpr int A_FLOATS = ROWS * LD;        // A_s^T[k'][i2], k' = 0..NP
    static constexpr int STAGE = 2 * A_FLOATS;        // + B[k'][j2], k' = 0..NP
    static constexpr int TASKS = NB * (NB + 1) * (NB + 2) / 6;
    static constexpr int THREADS = 128;
    // two stages plus the chunk table (one 32-bit entry per copied 16-byte chunk, <= 2*NP*CPR)
    static constexpr size_t SMEM = 2 * (size_t)STAGE * sizeof(float) + 2 * NP * CPR * sizeof(unsigned);
};

// shared offset (floats) of row r, column c (c a multiple of 4 for 16-byte accesses)
template <int NB>
__device__ __forceinline__ int r0_off(int r, int c)
{
    using Sh = R0Shape<NB>;
    if constexpr (Sh::SWZ) {
        const int cc = c >> 2;
        const int pc = cc ^ (cc >> 3) ^ (((r >> 3) & 3) << 1);
        return r * Sh::LD + (pc << 2) + (c & 3);
    } else {
        return r * Sh::LD + c;
    }
}

// task (bi, bj, kb) of each lane for Np = 64: 15 quarter-warps whose 128-bit shared loads of A
// and B hit 8 distinct bank groups (or one broadcast address) under r0_off's swizzle; lanes
// 120..127 idle.
__constant__ unsigned char c_r0_lane64[120][3] = {
    {0,2,0},{0,6,0},{0,5,0},{0,4,0},{0,0,0},{0,1,0},{0,7,0},{0,3,0},{1,4,1},{0,5,1},{0,7,1},{0,4,1},
    {0,6,1},{1,2,1},{1,7,1},{1,5,1},{0,2,2},{0,3,2},{2,5,2},{1,6,2},{1,5,2},{0,7,2},{1,2,2},{0,6,2},
    {2,7,2},{0,4,2},{2,3,2},{1,4,2},{2,2,2},{2,4,2},{2,6,2},{1,7,2},{2,3,3},{2,7,3},{1,7,3},{3,5,3},
    {3,7,3},{0,3,3},{1,4,3},{3,3,3},{2,5,3},{0,4,3},{0,7,3},{3,6,3},{2,6,3},{3,4,3},{2,4,3},{0,6,3},
    {2,7,4},{2,5,4},{0,7,4},{0,5,4},{1,7,4},{1,4,4},{1,6,4},{3,7,4},{0,6,4},{0,4,4},{4,4,4},{2,6,4},
    {3,4,4},{3,6,4},{2,4,4},{3,5,4},{5,6,5},{4,6,5},{2,7,5},{1,7,5},{5,7,5},{2,6,5},{1,6,5},{3,5,5},
    {0,6,5},{5,5,5},{3,6,5},{0,5,5},{2,5,5},{3,7,5},{4,7,5},{0,7,5},{4,7,6},{6,6,6},{6,7,6},{0,7,6},
    {0,6,6},{2,6,6},{3,6,6},{3,7,6},{0,7,7},{4,7,7},{3,7,7},{2,7,7},{1,7,7},{7,7,7},{5,7,7},{6,7,7},
    {0,2,1},{0,3,1},{1,3,1},{1,1,1},{0,1,1},{1,6,1},{1,3,2},{1,6,3},{0,5,2},{4,6,4},{2,7,6},{1,6,6},
    {1,7,6},{4,6,6},{5,6,6},{5,7,6},{1,3,3},{1,5,3},{0,5,3},{1,5,4},{4,5,4},{4,7,4},{1,5,5},{4,5,5}};

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem)
{
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// number of 16-byte chunks copied per k1: A_s rows 1..NP need cc with 4cc <= r; B rows 0..NP-1
// need cc with 4cc + 4 >= r (see r0_small_kernel)
__host__ __device__ constexpr int r0_a_chunks(int NP, int r) { return (r / 4 + 1) < NP / 4 ? r / 4 + 1 : NP / 4; }
__host__ __device__ constexpr int r0_b_first(int r) { return r <= 4 ? 0 : (r - 4 + 3) / 4; }

template <int NB>
__global__ void __launch_bounds__(128, 3)
r0_small_kernel(const R0Job *__restrict__ jobs, int njobs, const PairDesc *__restrict__ pairs,
                float *__restrict__ F, const float *__restrict__ FT, const float *__restrict__ S, int d)
{
    using Sh = R0Shape<NB>;
    constexpr int NP = Sh::NP, CPR = Sh::CPR;
    extern __shared__ __align__(16) float smem[];
    // chunk table after the two stages: (A or B, source offset in the tile, shared offset in the stage)
    unsigned *ctab = reinterpret_cast<unsigned *>(smem + 2 * Sh::STAGE);
    const int tid = threadIdx.x;
    int jid = blockIdx.x;
    if (jid >= njobs) return;

    // prologue (once per CTA): every shared slot -inf; chunks that only hold masked entries are
    // never copied, so their slots stay -inf for every job
    for (int q = tid * 4; q < 2 * Sh::STAGE; q += Sh::THREADS * 4)
        *reinterpret_cast<float4 *>(smem + q) = make_float4(NEG_INF, NEG_INF, NEG_INF, NEG_INF);
    int nchunks = 0;
    for (int r = 1; r <= NP; ++r) nchunks += r0_a_chunks(NP, r);
    for (int r = 0; r < NP; ++r) nchunks += CPR - r0_b_first(r);
    if (tid < 2 * NP) {  // one thread per copied row builds that row's entries
        int base = 0;
        const bool isA = tid < NP;
        const int row = isA ? tid + 1 : tid - NP;
        for (int r = 1; r <= (isA ? row - 1 : NP); ++r) base += r0_a_chunks(NP, r);
        if (!isA)
            for (int r = 0; r < row; ++r) base += CPR - r0_b_first(r);
        const int c0 = isA ? 0 : r0_b_first(row), c1 = isA ? r0_a_chunks(NP, row) : CPR;
        for (int cc = c0; cc < c1; ++cc) {
            const unsigned src = isA ? (row - 1) * NP + 4 * cc : row * NP + 4 * cc;
            const unsigned dst = (isA ? 0 : Sh::A_FLOATS) + r0_off<NB>(row, 4 * cc);
            ctab[base++] = (src << 16) | dst;
        }
    }
    __syncthreads();

    const long long tile = (long long)NP * NP;
    int bi = 0, bj = 0, kb = 0;
    const bool has_task = tid < Sh::TASKS;
    if constexpr (Sh::SWZ) {
        if (has_task) { bi = c_r0_lane64[tid][0]; bj = c_r0_lane64[tid][1]; kb = c_r0_lane64[tid][2]; }
    } else {
        int t = tid, found = 0;
        for (int a = 0; a < NB && !found; ++a)
            for (int b = a; b < NB && !found; ++b) {
                const int n = b - a + 1;
                if (t < n) { bi = a; bj = b; kb = a + t; found = 1; }
                else t -= n;
            }
    }
    const bool edge = has_task && kb == bj;

    // issues the copies of (job, k1) into stage
    auto load_stage = [&](int stage, const R0Job &jb, int k1) {
        const PairDesc pd = pairs[jb.pair];
        const int M = pd.M, j1 = jb.i1 + d;
        float *st = smem + stage * Sh::STAGE;
        const float *ga = FT + pd.F_off + cell_index(M, jb.i1, k1) * tile;  // column k of F(i1,k1)
        const float *gb = F + pd.F_off + cell_index(M, k1 + 1, j1) * tile;  // F(k1+1,j1)
        for (int e = tid; e < nchunks; e += Sh::THREADS) {
            const unsigned v = ctab[e];
            const unsigned dst = v & 0xffffu, src = v >> 16;
            cp_async16(st + dst, (dst < (unsigned)Sh::A_FLOATS ? ga : gb) + src);
        }
        const float *S1 = S + pd.S1_off;
        if (tid == 0) cp_async4(st + r0_off<NB>(0, 0), S1 + jb.i1 * M + k1);                               // R3 slot, i2 = 0
        if (tid == 1) cp_async4(st + Sh::A_FLOATS + r0_off<NB>(NP, NP - 4) + 3, S1 + (k1 + 1) * M + j1);  // R4 slot, j2 = NP-1
        cp_async_commit();
    };

    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = NEG_INF;

    R0Job job = jobs[jid];
    int k1 = job.k1a, stage = 0;
    load_stage(0, job, k1);
    while (true) {
        // the next (job, k1) item of this CTA, possibly in its next job
        R0Job njob = job;
        int njid = jid, nk1 = k1 + 1;
        if (nk1 >= job.k1b) {
            njid = jid + gridDim.x;
            if (njid < njobs) { njob = jobs[njid]; nk1 = njob.k1a; }
        }
        const bool has_next = njid < njobs;
        cp_async_wait<0>();
        // one barrier per item: it publishes this stage's copies and guarantees every thread has
        // finished the previous item, whose stage the next copies overwrite
        __syncthreads();
        if (has_next) load_stage(stage ^ 1, njob, nk1);
        const float *As = smem + stage * Sh::STAGE;
        const float *Bs = As + Sh::A_FLOATS;
        if (has_task) {
#pragma unroll
            for (int k = 0; k < 8; k += 2) {
                const int r = 8 * kb + k;
                const float4 a0 = *reinterpret_cast<const float4 *>(As + r0_off<NB>(r, 8 * bi));
                const float4 a1 = *reinterpret_cast<const float4 *>(As + r0_off<NB>(r, 8 * bi + 4));
                const float4 a2 = *reinterpret_cast<const float4 *>(As + r0_off<NB>(r + 1, 8 * bi));
                const float4 a3 = *reinterpret_cast<const float4 *>(As + r0_off<NB>(r + 1, 8 * bi + 4));
                const float4 b0 = *reinterpret_cast<const float4 *>(Bs + r0_off<NB>(r, 8 * bj));
                const float4 b1 = *reinterpret_cast<const float4 *>(Bs + r0_off<NB>(r, 8 * bj + 4));
                const float4 b2 = *reinterpret_cast<const float4 *>(Bs + r0_off<NB>(r + 1, 8 * bj));
                const float4 b3 = *reinterpret_cast<const float4 *>(Bs + r0_off<NB>(r + 1, 8 * bj + 4));
                const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
                const float aw[8] = {a2.x, a2.y, a2.z, a2.w, a3.x, a3.y, a3.z, a3.w};
                const float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
                const float bw[8] = {b2.x, b2.y, b2.z, b2.w, b3.x, b3.y, b3.z, b3.w};
#pragma unroll
                for (int i = 0; i < 8; ++i)
#pragma unroll
                    for (int j = 0; j < 8; ++j) acc[i][j] = fmax3(acc[i][j], av[i] + bv[j], aw[i] + bw[j]);
            }
            if (edge) {  // k' = 8bj+8: R4 of column j2 = 8bj+7
                const int r = 8 * bj + 8;
                const float4 a0 = *reinterpret_cast<const float4 *>(As + r0_off<NB>(r, 8 * bi));
                const float4 a1 = *reinterpret_cast<const float4 *>(As + r0_off<NB>(r, 8 * bi + 4));
                const float bs = Bs[r0_off<NB>(r, 8 * bj + 4) + 3];
                const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
#pragma unroll
                for (int i = 0; i < 8; ++i) acc[i][7] = fmaxf(acc[i][7], av[i] + bs);
            }
        }
        if (njid != jid || !has_next) {  // job done: merge its partial maxima into F(i1, i1+d)
            if (has_task) {
                const PairDesc pd = pairs[job.pair];
                int *out = reinterpret_cast<int *>(F + pd.F_off + cell_index(pd.M, job.i1, job.i1 + d) * tile);
#pragma unroll
                for (int i = 0; i < 8; ++i)
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const int i2 = 8 * bi + i, j2 = 8 * bj + j;
                        if (i2 <= j2 && j2 < pd.N) atomicMax(out + i2 * NP + j2, __float_as_int(acc[i][j]));
                        acc[i][j] = NEG_INF;
                    }
            }
        }
        if (!has_next) break;
        jid = njid;
        job = njob;
        k1 = nk1;
        stage ^= 1;
    }
}

// ------------------------------------------------------------------------------------------
// Finalize the outer cells of diagonal d (Np <= 64; 4 warps per cell): adds the candidates that
// do not come from R0/R3/R4 and runs the inner wavefront of R1/R2/SW2 in shared memory.
//   base  i1==j1 && i2==j2: inter(s1[i1], s2r[i2])            (assignment, eval_FTable :576)
//   S1(i1,j1)+S2(i2,j2)
//   SW2 = F(i1,j1,i2+1,j2-1)+intra(s2r[i2],s2r[j2]) if j2-i2>=4
//   R1 (:614-640) max_{k2} F(i1,j1,i2,k2)+S2(k2+1,j2); R2 (:641-667) max_{k2} S2(i2,k2)+F(i1,j1,k2+1,j2)
// F arrives holding max(R0,R3,R4,SW1) (or +0): SW1 = F(i1+1,j1-1,.)+intra(s1[i1],s1[j1])
// (V3/bpmax_outer_south_west.c:115-160) was stored into this cell's still-cleared table by the
// finalize of (i1+1, j1-1) two diagonals earlier, before any product touched it. Every literal-0
// candidate is covered because every value is >= +0. Writes F and FT: -inf outside the logical
// triangle and S1(i1,j1) on the subdiagonal (the R3/R4 slots of the product kernel).
// CTAs after the first njobs compute S1 on diagonal d+1 (V3/bpmax_verify.c:533-544), one warp
// per cell, from S1 diagonals <= d (S1 is cleared to 0 before the fill; j-i <= 3 stays 0).
// ------------------------------------------------------------------------------------------
struct CellJob {
    int pair, i1;
};

template <int NP>
struct FinShape {
    static constexpr int LD = NP + 4;             // 16-byte rows; conflict-free column walks
    static constexpr int TBL = NP * LD;           // one NP x NP table
    static constexpr size_t SMEM = 4 * (size_t)TBL * sizeof(float) + NP;
};

// The inner DP reads, for cell (i2,j2):  R1 = max_k F[i2][k] + S2[k+1][j2],  R2 = max_k S2[i2][k] + F[k+1][j2].
// Shared memory keeps F and S2 row-major plus shifted transposes FT1[j2][k] = F[k+1][j2] and
// ST1[j2][k] = S2[k+1][j2], so both are row-by-row scans with 16-byte loads. Every entry outside
// the logical triangles is -inf, so 4-aligned k chunks that overhang [i2, j2) only add -inf terms
// (k < i2 meets F[i2][k] or S2[i2][k]; k >= j2 meets ST1[j2][k] or FT1[j2][k]).
template <int NP>
__global__ void __launch_bounds__(128)
finalize_small_kernel(const CellJob *__restrict__ jobs, int njobs, const CellJob *__restrict__ s1jobs, int ns1,
                      const PairDesc *__restrict__ pairs, float *__restrict__ F, float *__restrict__ FT,
                      float *__restrict__ S, const uint8_t *__restrict__ bases, Weights W, int d)
{
    using Sh = FinShape<NP>;
    constexpr int LD = Sh::LD;
    extern __shared__ __align__(16) float fsm[];
    float *Fs = fsm, *FT1 = fsm + Sh::TBL, *Ss = fsm + 2 * Sh::TBL, *ST1 = fsm + 3 * Sh::TBL;
    uint8_t *sb = reinterpret_cast<uint8_t *>(fsm + 4 * Sh::TBL);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if ((int)blockIdx.x >= njobs) {  // S1 cells (i, i+d+1), one per warp
        const int q = ((int)blockIdx.x - njobs) * 4 + warp;
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
        if (lane == 0) S1[i * M + j] = fmaxf(S1[(i + 1) * M + (j - 1)] + score_w(W.w, s1[i], s1[j]), red);
        return;
    }
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
    const float s1v = S1[i1 * M + j1];
    for (int q = tid; q < NP; q += 128) sb[q] = q < N ? s2r[q] : 4;
    __syncthreads();  // sb is read by the staging loop (inter-strand base case)
    // staging: 16-byte loads of the accumulated F (max of R0, R3, R4, SW1) and of S2
    for (int q4 = tid; q4 < NP * NP / 4; q4 += 128) {
        const int r = (4 * q4) / NP, c0 = (4 * q4) % NP;
        const float4 a = *reinterpret_cast<const float4 *>(Fc + 4 * q4);
        const float4 b = *reinterpret_cast<const float4 *>(S2 + 4 * q4);
        const float av[4] = {a.x, a.y, a.z, a.w}, bv[4] = {b.x, b.y, b.z, b.w};
        float fv[4], sv[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int c = c0 + e;
            const bool valid = r <= c && c < N;
            sv[e] = valid ? bv[e] : NEG_INF;
            float v = NEG_INF;
            if (valid) v = (d == 0 && r == c) ? score_w(W.w + 6, s1[i1], sb[r]) : fmaxf(av[e], s1v + bv[e]);
            fv[e] = v;
            if (r >= 1) { FT1[c * LD + r - 1] = v; ST1[c * LD + r - 1] = sv[e]; }
        }
        *reinterpret_cast<float4 *>(Fs + r * LD + c0) = make_float4(fv[0], fv[1], fv[2], fv[3]);
        *reinterpret_cast<float4 *>(Ss + r * LD + c0) = make_float4(sv[0], sv[1], sv[2], sv[3]);
    }
    for (int c = tid; c < NP; c += 128) { FT1[c * LD + NP - 1] = NEG_INF; ST1[c * LD + NP - 1] = NEG_INF; }
    __syncthreads();
    for (int dd = 1; dd < N; ++dd) {
        const int cells = N - dd;  // <= 63 < 128: one pass
        const int g = min(32, 1 << (31 - __clz(128 / cells)));
        const int lane_g = tid & (g - 1);
        const int i2 = tid / g, j2 = i2 + dd;
        const bool act = i2 < cells;
        float r0 = NEG_INF, r1 = NEG_INF;
        if (act) {
            const float *fr = Fs + i2 * LD, *sr = Ss + i2 * LD, *ftr = FT1 + j2 * LD, *str = ST1 + j2 * LD;
            const int c_end = (j2 + 3) >> 2;
            for (int c = (i2 >> 2) + lane_g; c < c_end; c += g) {
                const float4 f = *reinterpret_cast<const float4 *>(fr + 4 * c);
                const float4 t = *reinterpret_cast<const float4 *>(str + 4 * c);
                const float4 s2 = *reinterpret_cast<const float4 *>(sr + 4 * c);
                const float4 u = *reinterpret_cast<const float4 *>(ftr + 4 * c);
                r0 = fmax3(r0, f.x + t.x, s2.x + u.x);
                r1 = fmax3(r1, f.y + t.y, s2.y + u.y);
                r0 = fmax3(r0, f.z + t.z, s2.z + u.z);
                r1 = fmax3(r1, f.w + t.w, s2.w + u.w);
            }
        }
        float red = fmaxf(r0, r1);
        for (int o = g >> 1; o > 0; o >>= 1) red = fmaxf(red, __shfl_xor_sync(0xffffffffu, red, o, g));
        if (act && lane_g == 0) {
            float v = fmaxf(Fs[i2 * LD + j2], red);
            if (dd >= 4) v = fmaxf(v, Fs[(i2 + 1) * LD + (j2 - 1)] + score_w(W.w, sb[i2], sb[j2]));
            Fs[i2 * LD + j2] = v;
            if (i2 >= 1) FT1[j2 * LD + i2 - 1] = v;
        }
        __syncthreads();
    }
    // SW1 candidate of cell (i1-1, j1+1), whose table nothing else has written yet
    const bool push = i1 >= 1 && j1 + 1 < M && d + 2 >= 4;
    const float wp = push ? score_w(W.w, s1[i1 - 1], s1[j1 + 1]) : 0.0f;
    float *Fn = push ? F + pd.F_off + cell_index(M, i1 - 1, j1 + 1) * tile : nullptr;
    for (int q4 = tid; q4 < NP * NP / 4; q4 += 128) {
        const int r = (4 * q4) / NP, c = (4 * q4) % NP;
        float4 v = *reinterpret_cast<const float4 *>(Fs + r * LD + c);
        if (push) {
            float4 u;
            u.x = (r <= c + 0 && c + 0 < N) ? v.x + wp : 0.0f;
            u.y = (r <= c + 1 && c + 1 < N) ? v.y + wp : 0.0f;
            u.z = (r <= c + 2 && c + 2 < N) ? v.z + wp : 0.0f;
            u.w = (r <= c + 3 && c + 3 < N) ? v.w + wp : 0.0f;
            *reinterpret_cast<float4 *>(Fn + 4 * q4) = u;
        }
        // S1(i1,j1) on the subdiagonal: the R3/R4 slots of the product kernel (never a logical cell)
        if (r == c + 1) v.x = s1v;
        if (r == c + 2) v.y = s1v;
        if (r == c + 3) v.z = s1v;
        if (r == c + 4) v.w = s1v;
        *reinterpret_cast<float4 *>(Fc + 4 * q4) = v;
        const float c0v = (r + 1 == c + 0) ? s1v : Fs[(c + 0) * LD + r];
        const float c1v = (r + 1 == c + 1) ? s1v : Fs[(c + 1) * LD + r];
        const float c2v = (r + 1 == c + 2) ? s1v : Fs[(c + 2) * LD + r];
        const float c3v = (r + 1 == c + 3) ? s1v : Fs[(c + 3) * LD + r];
        *reinterpret_cast<float4 *>(FTc + 4 * q4) = make_float4(c0v, c1v, c2v, c3v);
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
