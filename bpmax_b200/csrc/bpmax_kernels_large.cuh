// bpmax_kernels_large.cuh -- kernels for inner tables wider than 64 (Np = N rounded up to a
// multiple of 64). Same recurrence, layout and exactness argument as bpmax_kernels.cuh.
#pragma once
#include "bpmax_kernels.cuh"

namespace bpmax {

// ------------------------------------------------------------------------------------------
// Shared-memory stage of the wide product kernel: rows k' = 0..64 of the shifted A operand
// (A_s^T[k'][i2], 64 columns i2 of one output block) and of B (B[k'][j2], 64 columns j2), rows
// unpadded and XOR-swizzled per 16-byte chunk so that the task table below is conflict-free.
// ------------------------------------------------------------------------------------------
struct WideShape {
    static constexpr int NP = 64;
    static constexpr int LD = NP;                     // row stride (floats)
    static constexpr int ROWS = NP + 1;
    static constexpr int A_FLOATS = ROWS * LD;        // A_s^T[k'][i2], k' = 0..NP
    static constexpr int STAGE = 2 * A_FLOATS;        // + B[k'][j2], k' = 0..NP
    static constexpr int TASKS = 120;                 // (bi, bj, kb), bi <= kb <= bj < 8
    static constexpr size_t SMEM = 2 * (size_t)STAGE * sizeof(float);
};

// shared offset (floats) of row r, column c (c a multiple of 4 for 16-byte accesses)
__device__ __forceinline__ int wide_off(int r, int c)
{
    const int cc = c >> 2;
    const int pc = cc ^ (cc >> 3) ^ (((r >> 3) & 3) << 1);
    return r * WideShape::LD + (pc << 2) + (c & 3);
}

// task (bi, bj, kb) of each lane for a 64x64 diagonal output block: 15 quarter-warps whose 128-bit
// shared loads of A and B hit 8 distinct bank groups (or one broadcast address) under wide_off's
// swizzle; lanes 120..127 idle.
__constant__ unsigned char c_wide_lane[120][3] = {
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


// ------------------------------------------------------------------------------------------
// Rearranged copies of S2 (S2 over the reversed strand 2, V3/bpmax_verify.c:560-571) for the wide
// inner wavefronts (Np > 64): the masked S2M[i][k] = S2(i,k) if i <= k < N else -inf and
// ST1[j][k] = S2(k+1,j) if k+1 <= j < N else -inf (global-memory wavefront), and the
// triangular diagonal-major S2D: row e holds S2(i, i+e) for i = 0 .. Np-1-e (-inf where i+e >= N) at
// drow(Np, e) + i (shared-memory wavefront; T(Np) floats, half the square copy, so more of it stays
// in L1 beside the wavefront's shared-memory table). One CTA per pair; pairs of the cell-image widths
// have nothing to do.
// ------------------------------------------------------------------------------------------
__global__ void s2_aux_kernel(const PairDesc *__restrict__ pairs, float *__restrict__ S)
{
    const PairDesc pd = pairs[blockIdx.x];
    const int Np = pd.Np, N = pd.N;
    if (Np <= 64) return;
    const float *S2 = S + pd.S2_off;
    float *S2M = S + pd.S2m_off, *ST1 = S + pd.S2t_off, *S2D = S + pd.S2d_off;
    for (int q = threadIdx.x; q < Np * Np; q += blockDim.x) {
        const int r = q / Np, c = q % Np;
        S2M[q] = (r <= c && c < N) ? S2[q] : NEG_INF;
        ST1[q] = (c + 1 <= r && r < N) ? S2[(c + 1) * Np + r] : NEG_INF;
        if (c < Np - r) S2D[drow(Np, r) + c] = c + r < N ? S2[c * Np + c + r] : NEG_INF;  // r = e, c = i
    }
}

// ------------------------------------------------------------------------------------------
// R0 + R3 + R4 for Np = 64*NBk (row-major F and its transpose FT, Np x Np per outer cell). With
// A_s = F(i1,k1) shifted one column right (A_s[i2][k'] = F(i1,k1)[i2][k'-1], A_s[0][0] =
// S1(i1,k1)) and B = F(k1+1,j1) (S1(k1+1,j1) on its subdiagonal, guard row Np = S1(k1+1,j1) at
// column Np-1), R0, R3 and R4 are one triangular (max,+) product max_{k' in [i2, j2+1]}
// A_s[i2][k'] + B[k'][j2]. A job is one outer cell, one 64x64 output block (BI,BJ) and a k1
// range; it loops over the k' blocks KB in [BI, BJ]. Each stage holds rows k' = 64KB..64KB+64 of
// A_s (columns i2 of block BI, read from FT) and of B (columns j2 of block BJ) in WideShape's
// layout. Diagonal output blocks use the balanced triangular task table c_wide_lane; the
// other blocks give every thread one 8x8 micro-tile and half of the eight 8-wide k' sub-blocks
// (A is triangular in the stage KB == BI, B in the stage KB == BJ, dense in between).
// ------------------------------------------------------------------------------------------
struct R0JobL {
    int pair, i1, k1a, k1b, blk;  // blk = BI << 16 | BJ
};

__global__ void __launch_bounds__(128, 3)
r0_large_kernel(const R0JobL *__restrict__ jobs, int njobs, const PairDesc *__restrict__ pairs, float *__restrict__ F,
                const float *__restrict__ FT, const float *__restrict__ S, int d)
{
    using Sh = WideShape;
    constexpr int B = 64;
    extern __shared__ __align__(16) float smem[];
    const int tid = threadIdx.x;
    int jid = blockIdx.x;
    if (jid >= njobs) return;

    // issue the copies of (job, k1, KB) into stage
    auto load_item = [&](int stage, const R0JobL &jb, int k1, int KB) {
        const PairDesc pd = pairs[jb.pair];
        const int M = pd.M, Np = pd.Np, NBk = Np / B, j1 = jb.i1 + d;
        const int BI = jb.blk >> 16, BJ = jb.blk & 0xffff;
        const long long tile = (long long)Np * Np;
        float *st = smem + stage * Sh::STAGE;
        const float *ga = FT + pd.F_off + cell_index(M, jb.i1, k1) * tile;
        const float *gb = F + pd.F_off + cell_index(M, k1 + 1, j1) * tile;
        const float *S1 = S + pd.S1_off;
        for (int q = tid; q < 2 * (B + 1) * 16; q += 128) {
            const int which = q / ((B + 1) * 16), r = (q / 16) % (B + 1), cc = q % 16;
            const int kp = B * KB + r;  // global k'
            if (which == 0) {
                if (kp == 0) {  // A_s row 0: S1(i1,k1) at (0,0), -inf elsewhere
                    float4 v = make_float4(NEG_INF, NEG_INF, NEG_INF, NEG_INF);
                    if (BI == 0 && cc == 0) v.x = S1[jb.i1 * M + k1];
                    *reinterpret_cast<float4 *>(st + wide_off(r, 4 * cc)) = v;
                } else {
                    cp_async16(st + wide_off(r, 4 * cc), ga + (long long)(kp - 1) * Np + B * BI + 4 * cc);
                }
            } else {
                if (kp == Np) {  // guard row: S1(k1+1,j1) at (Np, Np-1), -inf elsewhere
                    float4 v = make_float4(NEG_INF, NEG_INF, NEG_INF, NEG_INF);
                    if (BJ == NBk - 1 && cc == 15) v.w = S1[(k1 + 1) * M + j1];
                    *reinterpret_cast<float4 *>(st + Sh::A_FLOATS + wide_off(r, 4 * cc)) = v;
                } else {
                    cp_async16(st + Sh::A_FLOATS + wide_off(r, 4 * cc), gb + (long long)kp * Np + B * BJ + 4 * cc);
                }
            }
        }
        cp_async_commit();
    };

    R0JobL job = jobs[jid];
    int BI = job.blk >> 16, BJ = job.blk & 0xffff;
    int k1 = job.k1a, KB = BI, stage = 0;
    // per-job thread mapping (diagonal vs off-diagonal output block)
    int bi = 0, bj = 0, kb = 0, h = 0;
    bool has_task = false;
    auto map_threads = [&]() {
        if (BI == BJ) {
            has_task = tid < WideShape::TASKS;
            if (has_task) { bi = c_wide_lane[tid][0]; bj = c_wide_lane[tid][1]; kb = c_wide_lane[tid][2]; }
        } else {
            has_task = true;
            const int m = tid & 63;
            bi = m >> 3;
            bj = m & 7;
            h = tid >> 6;
        }
    };
    map_threads();
    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = NEG_INF;

    auto step8 = [&](const float *As, const float *Bs, int kbl) {
#pragma unroll
        for (int k = 0; k < 8; k += 2) {
            const int r = 8 * kbl + k;
            const float4 a0 = *reinterpret_cast<const float4 *>(As + wide_off(r, 8 * bi));
            const float4 a1 = *reinterpret_cast<const float4 *>(As + wide_off(r, 8 * bi + 4));
            const float4 a2 = *reinterpret_cast<const float4 *>(As + wide_off(r + 1, 8 * bi));
            const float4 a3 = *reinterpret_cast<const float4 *>(As + wide_off(r + 1, 8 * bi + 4));
            const float4 b0 = *reinterpret_cast<const float4 *>(Bs + wide_off(r, 8 * bj));
            const float4 b1 = *reinterpret_cast<const float4 *>(Bs + wide_off(r, 8 * bj + 4));
            const float4 b2 = *reinterpret_cast<const float4 *>(Bs + wide_off(r + 1, 8 * bj));
            const float4 b3 = *reinterpret_cast<const float4 *>(Bs + wide_off(r + 1, 8 * bj + 4));
            const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            const float aw[8] = {a2.x, a2.y, a2.z, a2.w, a3.x, a3.y, a3.z, a3.w};
            const float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
            const float bw[8] = {b2.x, b2.y, b2.z, b2.w, b3.x, b3.y, b3.z, b3.w};
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] = fmax3(acc[i][j], av[i] + bv[j], aw[i] + bw[j]);
        }
    };
    auto edge_step = [&](const float *As, const float *Bs) {  // k' = 8bj+8 (local): R4 of column 8bj+7
        const int r = 8 * bj + 8;
        const float4 a0 = *reinterpret_cast<const float4 *>(As + wide_off(r, 8 * bi));
        const float4 a1 = *reinterpret_cast<const float4 *>(As + wide_off(r, 8 * bi + 4));
        const float bs = Bs[wide_off(r, 8 * bj + 4) + 3];
        const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
#pragma unroll
        for (int i = 0; i < 8; ++i) acc[i][7] = fmaxf(acc[i][7], av[i] + bs);
    };

    load_item(0, job, k1, KB);
    while (true) {
        // next item: KB advances fastest, then k1, then the job
        R0JobL njob = job;
        int njid = jid, nk1 = k1, nKB = KB + 1;
        if (nKB > BJ) {
            nKB = -1;
            nk1 = k1 + 1;
            if (nk1 >= job.k1b) {
                njid = jid + gridDim.x;
                if (njid < njobs) { njob = jobs[njid]; nk1 = njob.k1a; }
            }
        }
        const bool has_next = njid < njobs;
        if (nKB < 0) nKB = has_next ? (njob.blk >> 16) : 0;
        cp_async_wait<0>();
        __syncthreads();
        if (has_next) load_item(stage ^ 1, njob, nk1, nKB);
        const float *As = smem + stage * Sh::STAGE;
        const float *Bs = As + Sh::A_FLOATS;
        if (has_task) {
            if (BI == BJ) {
                step8(As, Bs, kb);
                if (kb == bj) edge_step(As, Bs);
            } else {
                int lo = 4 * h, hi = 4 * h + 4;
                if (KB == BI) lo = max(lo, bi);
                if (KB == BJ) hi = min(hi, bj + 1);
                for (int kbl = lo; kbl < hi; ++kbl) step8(As, Bs, kbl);
                if (KB == BJ && bj >= 4 * h && bj < 4 * h + 4) edge_step(As, Bs);
            }
        }
        if (njid != jid || !has_next) {  // job done: merge its partial maxima into F(i1, i1+d)
            if (has_task) {
                const PairDesc pd = pairs[job.pair];
                const long long tile = (long long)pd.Np * pd.Np;
                int *out = reinterpret_cast<int *>(F + pd.F_off + cell_index(pd.M, job.i1, job.i1 + d) * tile);
#pragma unroll
                for (int i = 0; i < 8; ++i)
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const int i2 = B * BI + 8 * bi + i, j2 = B * BJ + 8 * bj + j;
                        if (i2 <= j2 && j2 < pd.N) atomicMax(out + (long long)i2 * pd.Np + j2, __float_as_int(acc[i][j]));
                        acc[i][j] = NEG_INF;
                    }
            }
        }
        if (!has_next) break;
        if (njid != jid) {
            job = njob;
            BI = job.blk >> 16;
            BJ = job.blk & 0xffff;
            map_threads();
        }
        jid = njid;
        k1 = nk1;
        KB = nKB;
        stage ^= 1;
    }
}

// ------------------------------------------------------------------------------------------
// Inner wavefront for Np > FIN_WIDE_MAX_NP (row-major F and its transpose FT, Np x Np per outer
// cell, in global memory), spread over the whole GPU and blocked in 64x64 tiles. The outer cells of
// diagonal d are finalized together. Tile (I, J) of F (rows 64I.., columns 64J..) needs
//   R1  F[i2][k] + S2(k+1, j2), k in [i2, j2): k < 64J lies in the finished tiles (I, K), K < J;
//       k >= 64J in the tile itself
//   R2  S2(i2, k) + F[k+1][j2], k+1 in (i2, j2]: k+1 >= 64(I+1) lies in the finished tiles (K, J),
//       K > I; k+1 < 64(I+1) in the tile itself
// so the tiles are done by tile diagonal t = J - I: first the terms over finished tiles as max-plus
// tile products (large_tile_product_kernel, t >= 1), then the tile's own terms, SW2 and its final
// values by a local wavefront over the tile's diagonals b - a in shared memory
// (large_tile_local_kernel). Every launch covers the tiles of diagonal t of every outer cell, and
// the launch boundaries are the only barriers (2 Np/64 + 1 launches per outer diagonal). The
// entries below the diagonal and past N are -inf in F and in the masked copies S2M, ST1, so the
// products need no bounds of their own. (One CTA per outer cell walking all N-1 inner steps used
// at most M-d SMs: a 16x3000 fill took 87 s in it.) Same candidates as finalize_small_kernel: base
// inter, S1+S2, SW1 (already in F, pushed two diagonals earlier), SW2, R1, R2.
//   large_init_kernel          start values of every entry of F, and FT, through 32x32 tiles
//   large_tile_product_kernel  the R1/R2 terms over finished tiles, merged into F
//   large_tile_local_kernel    the tile's own R1/R2 terms and SW2, then F and FT of the tile
//   large_final_kernel         the SW1 push into (i1-1, j1+1), S1 on the subdiagonal of F and the
//                              superdiagonal of FT; CTAs after the cells' compute S1 on diagonal d+1
// ------------------------------------------------------------------------------------------
constexpr int LARGE_FINAL_CHUNK = 8192;  // table entries per CTA of large_final_kernel

// grid (Np/32)^2 tiles x cells, block 32 x 8
__global__ void __launch_bounds__(256)
large_init_kernel(const CellJob *__restrict__ jobs, const PairDesc *__restrict__ pairs, float *__restrict__ F,
                  float *__restrict__ FT, const float *__restrict__ S, const uint8_t *__restrict__ bases, Weights W,
                  int d)
{
    __shared__ float tl[32][33];
    const CellJob job = jobs[blockIdx.y];
    const PairDesc pd = pairs[job.pair];
    const int M = pd.M, N = pd.N, Np = pd.Np, i1 = job.i1, j1 = i1 + d;
    const int nt = Np >> 5, tr = (int)blockIdx.x / nt, tc = (int)blockIdx.x % nt;
    const long long tile = (long long)Np * Np;
    float *Fc = F + pd.F_off + cell_index(M, i1, j1) * tile;
    float *FTc = FT + pd.F_off + cell_index(M, i1, j1) * tile;
    const float *S2 = S + pd.S2_off;
    const float s1v = S[pd.S1_off + i1 * M + j1];
    const uint8_t *s1 = bases + pd.seq1_off, *s2r = bases + pd.seq2_off;
    const int x = threadIdx.x;
    for (int y = threadIdx.y; y < 32; y += 8) {
        const int r = 32 * tr + y, c = 32 * tc + x;
        const long long q = (long long)r * Np + c;
        float v = NEG_INF;
        if (r <= c && c < N) v = (d == 0 && r == c) ? score_w(W.w + 6, s1[i1], s2r[r]) : fmaxf(Fc[q], s1v + S2[q]);
        Fc[q] = v;
        tl[y][x] = v;
    }
    __syncthreads();
    for (int y = threadIdx.y; y < 32; y += 8)  // FT[c][r] = F[r][c]: row 32tc+y, columns 32tr+x
        FTc[(long long)(32 * tc + y) * Np + 32 * tr + x] = tl[x][y];
}

constexpr int LT = 64;       // tile side
constexpr int LT_LD = 66;    // shared row stride of the product's operand slabs (8-byte pairs, conflict-free)
constexpr int LT_LD1 = 65;   // shared row stride of the local wavefront's tables
constexpr size_t LARGE_LOCAL_SMEM = 3 * LT * LT_LD1 * sizeof(float);

// grid (NT - t) x cells, 256 threads (16 x 16): tile (I, I+t) of each outer cell. Thread (tx, ty)
// owns outputs a = ty + 16u, b = tx + 16v (u, v < 4). Slabs of 64 k: R1 with A = F rows i2 and
// B = ST1 rows j2 over k in [64K, 64K+64), K = I .. J-1; R2 with A = S2M rows i2 over
// k = 64K-1 .. 64K+62 and B = FT rows j2 over k+1 = 64K .. 64K+63, K = I+1 .. J. Candidates are added
// in k pairs: (A[a][k], A[a][k+1]) + (B[b][k], B[b][k+1]), both neighbouring words of a slab row.
__global__ void __launch_bounds__(256)
large_tile_product_kernel(const CellJob *__restrict__ jobs, const PairDesc *__restrict__ pairs, float *__restrict__ F,
                          const float *__restrict__ FT, const float *__restrict__ S, int d, int t)
{
    __shared__ __align__(16) float As[LT * LT_LD];
    __shared__ __align__(16) float Bs[LT * LT_LD];
    const CellJob job = jobs[blockIdx.y];
    const PairDesc pd = pairs[job.pair];
    const int M = pd.M, N = pd.N, Np = pd.Np, I = (int)blockIdx.x, J = I + t;
    if (LT * I >= N || LT * J >= N) return;  // the tile lies past the table (CTA-uniform)
    const long long tile = (long long)Np * Np, cell = cell_index(M, job.i1, job.i1 + d);
    float *Fc = F + pd.F_off + cell * tile;
    const float *FTc = FT + pd.F_off + cell * tile;
    const float *S2M = S + pd.S2m_off, *ST1 = S + pd.S2t_off;
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    float acc[4][4];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[u][v] = NEG_INF;
    // slab q: q < t is R1 with K = I + q, q >= t is R2 with K = I + 1 + (q - t)
    for (int q = 0; q < 2 * t; ++q) {
        const bool r1 = q < t;
        const int K = r1 ? I + q : I + 1 + (q - t);
        const float *A = r1 ? Fc : S2M;            // rows 64I + a
        const float *B = r1 ? ST1 : FTc;           // rows 64J + b
        const int ka = r1 ? LT * K : LT * K - 1;   // first column of the A slab
        const int kb = LT * K;                     // first column of the B slab
        __syncthreads();  // the previous slab is no longer read
        for (int e = tid; e < LT * LT; e += 256) {
            const int r = e >> 6, c = e & 63;
            As[r * LT_LD + c] = A[(long long)(LT * I + r) * Np + ka + c];
            Bs[r * LT_LD + c] = B[(long long)(LT * J + r) * Np + kb + c];
        }
        __syncthreads();
#pragma unroll 4
        for (int k = 0; k < LT; k += 2) {
            float2 av[4], bv[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) av[u] = *reinterpret_cast<const float2 *>(As + (ty + 16 * u) * LT_LD + k);
#pragma unroll
            for (int v = 0; v < 4; ++v) bv[v] = *reinterpret_cast<const float2 *>(Bs + (tx + 16 * v) * LT_LD + k);
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    const float2 sm = __fadd2_rn(av[u], bv[v]);
                    acc[u][v] = fmax3(acc[u][v], sm.x, sm.y);
                }
        }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const int i2 = LT * I + ty + 16 * u, j2 = LT * J + tx + 16 * v;
            if (i2 <= j2 && j2 < N) {
                float *f = Fc + (long long)i2 * Np + j2;
                *f = fmaxf(*f, acc[u][v]);
            }
        }
}

// grid (NT - t) x cells, 256 threads: tile (I, I+t) of each outer cell, local coordinates
// (a, b) = (i2 - 64I, j2 - 64J). An entry depends on the entries left of it in its tile row (R1),
// below it in its tile column (R2) and at (a+1, b-1) (SW2), so the tile's diagonals b - a are done
// in increasing order, one CTA barrier each, 4 to 32 threads per entry:
//   R1  T[a][b'] + S2(64J+b'+1, 64J+b),   b' < b     (ST1 block rows 64J+b, columns 64J+b')
//   R2  S2(64I+a, 64I+a'-1) + T[a'][b],   a' > a     (S2M block rows 64I+a, columns 64I+a'-1)
// (on a diagonal tile the terms outside b' >= a, a' <= b meet a -inf entry below the diagonal).
// T starts with F's values after the tile product (start values, SW1, R0/R3/R4, terms over
// finished tiles); at the end F and FT take the tile.
__global__ void __launch_bounds__(256)
large_tile_local_kernel(const CellJob *__restrict__ jobs, const PairDesc *__restrict__ pairs, float *__restrict__ F,
                        float *__restrict__ FT, const float *__restrict__ S, const uint8_t *__restrict__ bases,
                        Weights W, int d, int t)
{
    extern __shared__ float ltl[];      // LARGE_LOCAL_SMEM bytes
    float *Tt = ltl;                    // the tile
    float *Sj = ltl + LT * LT_LD1;      // Sj[b][b'] = ST1[64J+b][64J+b'] = S2(64J+b'+1, 64J+b)
    float *Si = ltl + 2 * LT * LT_LD1;  // Si[a][c] = S2M[64I+a][64I+c] = S2(64I+a, 64I+c)
    const CellJob job = jobs[blockIdx.y];
    const PairDesc pd = pairs[job.pair];
    const int M = pd.M, N = pd.N, Np = pd.Np, I = (int)blockIdx.x, J = I + t;
    if (LT * I >= N || LT * J >= N) return;  // the tile lies past the table (CTA-uniform)
    const long long tile = (long long)Np * Np, cell = cell_index(M, job.i1, job.i1 + d);
    float *Fc = F + pd.F_off + cell * tile;
    float *FTc = FT + pd.F_off + cell * tile;
    const float *S2M = S + pd.S2m_off, *ST1 = S + pd.S2t_off;
    const uint8_t *s2r = bases + pd.seq2_off;
    const int tid = threadIdx.x;
    for (int e = tid; e < LT * LT; e += 256) {
        const int r = e >> 6, c = e & 63;
        Tt[r * LT_LD1 + c] = Fc[(long long)(LT * I + r) * Np + LT * J + c];
        Sj[r * LT_LD1 + c] = ST1[(long long)(LT * J + r) * Np + LT * J + c];
        Si[r * LT_LD1 + c] = S2M[(long long)(LT * I + r) * Np + LT * I + c];
    }
    __syncthreads();
    for (int l = (t == 0 ? 1 : -(LT - 1)); l < LT; ++l) {
        // the 64 - |l| entries of tile diagonal l, G threads each (G = 4 .. 32, as many as 256 allow):
        // entries far from the tile's main diagonal hold the most terms and the fewest entries
        const int E = LT - (l < 0 ? -l : l);
        const int lg = E > 32 ? 2 : (E > 16 ? 3 : (E > 8 ? 4 : 5)), G = 1 << lg;
        const int g = tid & (G - 1), slot = tid >> lg;
        const int a = l >= 0 ? slot : slot - l, b = a + l;  // entry slot of tile diagonal l
        const int i2 = LT * I + a, j2 = LT * J + b;
        const bool act = a < LT && b < LT && b >= 0 && i2 <= j2 && j2 < N;
        float red = NEG_INF, red1 = NEG_INF;  // two chains of maxima per thread
        if (act) {
            int bp = g;
            for (; bp + G < b; bp += 2 * G) {
                red = fmaxf(red, Tt[a * LT_LD1 + bp] + Sj[b * LT_LD1 + bp]);
                red1 = fmaxf(red1, Tt[a * LT_LD1 + bp + G] + Sj[b * LT_LD1 + bp + G]);
            }
            if (bp < b) red = fmaxf(red, Tt[a * LT_LD1 + bp] + Sj[b * LT_LD1 + bp]);
            int ap = a + 1 + g;
            for (; ap + G < LT; ap += 2 * G) {
                red = fmaxf(red, Si[a * LT_LD1 + ap - 1] + Tt[ap * LT_LD1 + b]);
                red1 = fmaxf(red1, Si[a * LT_LD1 + ap + G - 1] + Tt[(ap + G) * LT_LD1 + b]);
            }
            if (ap < LT) red = fmaxf(red, Si[a * LT_LD1 + ap - 1] + Tt[ap * LT_LD1 + b]);
        }
        red = fmaxf(red, red1);
        for (int o = G >> 1; o > 0; o >>= 1) red = fmaxf(red, __shfl_xor_sync(0xffffffffu, red, o));  // G is CTA-uniform
        if (act && g == 0) {
            float v = fmaxf(Tt[a * LT_LD1 + b], red);
            if (j2 - i2 >= 4) {
                // SW2 entry (i2+1, j2-1): in the tile, or in a finished tile below or to the left
                const float sw = (a + 1 < LT && b >= 1) ? Tt[(a + 1) * LT_LD1 + b - 1]
                                                        : Fc[(long long)(i2 + 1) * Np + (j2 - 1)];
                v = fmaxf(v, sw + score_w(W.w, s2r[i2], s2r[j2]));
            }
            Tt[a * LT_LD1 + b] = v;
        }
        __syncthreads();
    }
    for (int e = tid; e < LT * LT; e += 256) {
        const int r = e >> 6, c = e & 63;
        Fc[(long long)(LT * I + r) * Np + LT * J + c] = Tt[r * LT_LD1 + c];
        FTc[(long long)(LT * J + r) * Np + LT * I + c] = Tt[c * LT_LD1 + r];
    }
}

// CTAs [0, ncells * chunks): entries [chunk * LARGE_FINAL_CHUNK, ...) of one outer cell; after them,
// one warp per S1 cell (i, i+d+1)
__global__ void __launch_bounds__(256)
large_final_kernel(const CellJob *__restrict__ jobs, int ncells, int chunks, const CellJob *__restrict__ s1jobs,
                   int ns1, const PairDesc *__restrict__ pairs, float *__restrict__ F, float *__restrict__ FT,
                   float *__restrict__ S, const uint8_t *__restrict__ bases, Weights W, int d)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int b = (int)blockIdx.x;
    if (b >= ncells * chunks) {  // S1 cells (i, i+d+1), one per warp
        const int q = (b - ncells * chunks) * 8 + warp;
        if (q >= ns1) return;
        const CellJob job = s1jobs[q];
        const PairDesc pd = pairs[job.pair];
        const int M = pd.M, i = job.i1, j = i + d + 1;
        float *S1 = S + pd.S1_off;
        if (j - i <= 3) return;
        const uint8_t *s1 = bases + pd.seq1_off;
        float red = NEG_INF;
        for (int k = i + lane; k < j; k += 32) red = fmaxf(red, S1[i * M + k] + S1[(k + 1) * M + j]);
        for (int o = 16; o > 0; o >>= 1) red = fmaxf(red, __shfl_xor_sync(0xffffffffu, red, o));
        if (lane == 0) S1[i * M + j] = fmaxf(S1[(i + 1) * M + (j - 1)] + score_w(W.w, s1[i], s1[j]), red);
        return;
    }
    const int ch = b % chunks;
    const CellJob job = jobs[b / chunks];
    const PairDesc pd = pairs[job.pair];
    const int M = pd.M, N = pd.N, Np = pd.Np, i1 = job.i1, j1 = i1 + d;
    const long long tile = (long long)Np * Np;
    float *Fc = F + pd.F_off + cell_index(M, i1, j1) * tile;
    float *FTc = FT + pd.F_off + cell_index(M, i1, j1) * tile;
    const float s1v = S[pd.S1_off + i1 * M + j1];
    // SW1 candidate of cell (i1-1, j1+1), whose table nothing else has written yet (entries r <= c;
    // the subdiagonal written below is not among them)
    if (i1 >= 1 && j1 + 1 < M && d + 2 >= 4) {
        const uint8_t *s1 = bases + pd.seq1_off;
        const float wp = score_w(W.w, s1[i1 - 1], s1[j1 + 1]);
        float *Fn = F + pd.F_off + cell_index(M, i1 - 1, j1 + 1) * tile;
        const long long q1 = min(tile, (long long)(ch + 1) * LARGE_FINAL_CHUNK);
        for (long long q = (long long)ch * LARGE_FINAL_CHUNK + tid; q < q1; q += 256) {
            const int r = (int)(q / Np), c = (int)(q % Np);
            Fn[q] = (r <= c && c < N) ? Fc[q] + wp : 0.0f;
        }
    }
    if (ch == 0)  // S1(i1,j1) on the subdiagonal of F (and the superdiagonal of FT): the R3/R4 slots
        for (int r = 1 + tid; r < Np; r += 256) {
            Fc[(long long)r * Np + r - 1] = s1v;
            FTc[(long long)(r - 1) * Np + r] = s1v;
        }
}

// ------------------------------------------------------------------------------------------
// S2 (V3/bpmax_verify.c:560-571) of one pair with Np > FIN_WIDE_MAX_NP, one launch per diagonal d of
// its wavefront (single_strand_kernel's one CTA per pair took 2.2 s at N = 3000), one warp per cell.
// The column operand S2(k+1, j) is read from ST1[j][k], which the same launches fill as cells become
// final (s2_aux_kernel rewrites ST1 completely afterwards); S starts at 0, so ST1 holds the 0 of
// every cell with j-i <= 3.
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
s2_diag_kernel(const PairDesc *__restrict__ pairs, int p, const uint8_t *__restrict__ bases, float *__restrict__ S,
               Weights W, int d)
{
    const PairDesc pd = pairs[p];
    const int L = pd.N, ld = pd.Np;
    const int i = (int)blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (i >= L - d) return;
    const int j = i + d;
    float *T = S + pd.S2_off, *TT = S + pd.S2t_off;
    const uint8_t *s = bases + pd.seq2_off;
    float r0 = NEG_INF, r1 = NEG_INF;
    int k = i + lane;
    for (; k + 32 < j; k += 64) {
        r0 = fmaxf(r0, T[(long long)i * ld + k] + TT[(long long)j * ld + k]);
        r1 = fmaxf(r1, T[(long long)i * ld + k + 32] + TT[(long long)j * ld + k + 32]);
    }
    if (k < j) r0 = fmaxf(r0, T[(long long)i * ld + k] + TT[(long long)j * ld + k]);
    float red = fmaxf(r0, r1);
    for (int o = 16; o > 0; o >>= 1) red = fmaxf(red, __shfl_xor_sync(0xffffffffu, red, o));
    if (lane == 0) {
        const float v = fmaxf(T[(long long)(i + 1) * ld + (j - 1)] + score_w(W.w, s[i], s[j]), red);
        T[(long long)i * ld + j] = v;
        if (i >= 1) TT[(long long)j * ld + i - 1] = v;
    }
}

// ------------------------------------------------------------------------------------------
// Finalize for 64 < Np <= FIN_WIDE_MAX_NP (tables stored as tile images, bpmax_kernels.cuh): same
// candidates and same results as the row-major tables' tile wavefront, pushed forward in
// shared memory. The CTA keeps the cell's inner table diagonal-major and triangular,
// D[e][i2] = F[i2][i2+e] (T(Np) floats), each open entry holding its running maximum. When inner
// diagonal e is final, every open cell (e2 > e) takes its two candidates that read diagonal e,
//   R1 with k2 = i2+e:    F[i2][i2+e] + S2(i2+e+1, j2)
//   R2 with k2 = j2-e-1:  S2(i2, j2-e-1) + F[j2-e][j2]
// and the cells of diagonal e+1 become final after SW2. Warp w takes the diagonals e2 = e+1+w,
// e+1+w+32, ...; its lanes take consecutive i2, so both S2 reads are one coalesced line of the
// diagonal-major copy and the D reads are conflict-free. One CTA barrier per inner diagonal. The
// tile images (blocks, S1 pieces of the diagonal tiles, halo pieces of the dense tiles) are written
// once, at the end, four columns of one block row per thread and step.
// CTAs after the first njobs compute S1 on diagonal d+1, one warp per cell.
// ------------------------------------------------------------------------------------------
constexpr int FIN_WIDE_THREADS = 1024;
constexpr int FIN_WIDE_MAX_NP = 320;  // T(320) floats = 205,440 bytes of shared memory
static_assert(FIN_WIDE_MAX_NP == WIDE_TILE_MAX_NP, "tables wider than the tile images are the row-major ones");

__host__ __device__ constexpr size_t fin_wide_smem(int Np) { return (size_t)Np * (Np + 1) / 2 * 4 + Np; }

__global__ void __launch_bounds__(FIN_WIDE_THREADS)
finalize_wide_kernel(const CellJob *__restrict__ jobs, int njobs, const CellJob *__restrict__ s1jobs, int ns1,
                     const PairDesc *__restrict__ pairs, float *__restrict__ F, float *__restrict__ S,
                     const uint8_t *__restrict__ bases, Weights W, int d)
{
    constexpr int NT = FIN_WIDE_THREADS, WARPS = NT / 32;
    extern __shared__ __align__(16) float fwd[];
    __shared__ float wsh[12];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid < 12) wsh[tid] = W.w[tid];
    __syncthreads();
    if ((int)blockIdx.x >= njobs) {  // S1 cells (i, i+d+1), one per warp
        const int q = ((int)blockIdx.x - njobs) * WARPS + warp;
        if (q >= ns1) return;
        const CellJob job = s1jobs[q];
        const PairDesc pd = pairs[job.pair];
        const int M = pd.M, i = job.i1, j = i + d + 1;
        float *S1 = S + pd.S1_off;
        if (j - i <= 3) return;
        const uint8_t *s1 = bases + pd.seq1_off;
        float red = NEG_INF;
        for (int k = i + lane; k < j; k += 32) red = fmaxf(red, S1[i * M + k] + S1[(k + 1) * M + j]);
        for (int o = 16; o > 0; o >>= 1) red = fmaxf(red, __shfl_xor_sync(0xffffffffu, red, o));
        if (lane == 0) S1[i * M + j] = fmaxf(S1[(i + 1) * M + (j - 1)] + score_w(wsh, s1[i], s1[j]), red);
        return;
    }
    const CellJob job = jobs[blockIdx.x];
    const PairDesc pd = pairs[job.pair];
    const int M = pd.M, N = pd.N, Np = pd.Np, NTL = Np >> 6, i1 = job.i1, j1 = i1 + d;
    const long long CELL = wide_cell_floats(NTL);
    float *Fc = F + pd.F_off + cell_index(M, i1, j1) * CELL;
    const float *S1 = S + pd.S1_off;
    const float *S2 = S + pd.S2_off;
    const float *S2D = S + pd.S2d_off;
    const uint8_t *s1 = bases + pd.seq1_off;
    float *D = fwd;
    uint8_t *sb = reinterpret_cast<uint8_t *>(fwd + Np * (Np + 1) / 2);
    for (int r = tid; r < Np; r += NT) sb[r] = r < N ? bases[pd.seq2_off + r] : 4;
    const float s1v = S1[i1 * M + j1];
    __syncthreads();
    // start values: max(accumulated, S1+S2), or the inter-strand base on the diagonal of the
    // diagonal cells
    for (int q = tid; q < Np * Np; q += NT) {
        const int r = q / Np, c = q % Np;
        if (r <= c && c < N)
            D[drow(Np, c - r) + r] =
                (d == 0 && r == c) ? score_w(wsh + 6, s1[i1], sb[r]) : fmaxf(Fc[wide_pos(NTL, r, c)], s1v + S2[q]);
    }
    __syncthreads();
    for (int e = 0; e + 1 < N; ++e) {
        const float *De = D + drow(Np, e);
        for (int e2 = e + 1 + warp; e2 < N; e2 += WARPS) {
            float *Dw = D + drow(Np, e2);
            const float *S2r = S2D + drow(Np, e2 - e - 1);
            const bool fin = e2 == e + 1 && e2 >= 4;
            const float *Dp = D + drow(Np, max(e2 - 2, 0)) + 1;
            for (int i2 = lane; i2 < N - e2; i2 += 32) {
                const int j2 = i2 + e2;
                float v = fmax3(Dw[i2], De[i2] + S2r[i2 + e + 1], S2r[i2] + De[j2 - e]);
                if (fin) v = fmaxf(v, Dp[i2] + score_w(wsh, sb[i2], sb[j2]));
                Dw[i2] = v;
            }
        }
        __syncthreads();
    }
    // the tile images: the logical triangle, S1(i1,j1) on the subdiagonal, -inf elsewhere; the S1
    // pieces of the diagonal tiles and the halo pieces of the dense ones; and the SW1 candidate of
    // cell (i1-1, j1+1), whose table nothing else has written yet (blocks only)
    const bool push = i1 >= 1 && j1 + 1 < M && d + 2 >= 4;
    const float wp = push ? score_w(wsh, s1[i1 - 1], s1[j1 + 1]) : 0.0f;
    float *Fn = push ? F + pd.F_off + cell_index(M, i1 - 1, j1 + 1) * CELL : nullptr;
    auto val = [&](int r, int c) {  // stored value of entry (r, c), r <= c + 1
        return (r <= c && c < N) ? D[drow(Np, c - r) + r] : (r == c + 1 ? s1v : NEG_INF);
    };
    for (int I = 0; I < NTL; ++I)
        for (int J = I; J < NTL; ++J) {
            const long long to = wide_tile_off(NTL, I, J);
            const int nblk = I == J ? 36 : 64;
            for (int q4 = tid; q4 < nblk * 16 + 16; q4 += NT) {
                if (q4 >= nblk * 16) {  // the closing piece of block column bj: S1 piece or halo piece
                    const int bj = (q4 - nblk * 16) >> 1, h = q4 & 1;
                    const int cb = I == J ? c_img_colbase[8][bj] : c_wide_dense_colbase[bj];
                    float v[4];
#pragma unroll
                    for (int t = 0; t < 4; ++t)
                        v[t] = I == J ? ((h == 1 && t == 3) ? s1v : NEG_INF) : val(64 * I + 64, 64 * J + 8 * bj + 4 * h + t);
                    *reinterpret_cast<float4 *>(Fc + to + 4 * (cb + 17 * (I == J ? bj + 1 : 8)) + 4 * h) =
                        make_float4(v[0], v[1], v[2], v[3]);
                    continue;
                }
                int bi, bj;
                if (I == J) {
                    blk_decode(8, q4 >> 4, bi, bj);
                } else {
                    bi = (q4 >> 4) & 7;
                    bj = q4 >> 7;
                }
                const int r = 64 * I + 8 * bi + ((q4 & 15) >> 1), c0 = 64 * J + 8 * bj + 4 * (q4 & 1);
                float v[4], u[4];
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    const int c = c0 + t;
                    v[t] = val(r, c);
                    u[t] = (r <= c && c < N) ? v[t] + wp : 0.0f;
                }
                const long long o = to + 4 * ((I == J ? c_img_colbase[8][bj] : c_wide_dense_colbase[bj]) + 17 * bi) +
                                    4 * (q4 & 15);
                if (push) *reinterpret_cast<float4 *>(Fn + o) = make_float4(u[0], u[1], u[2], u[3]);
                *reinterpret_cast<float4 *>(Fc + o) = make_float4(v[0], v[1], v[2], v[3]);
            }
        }
}

}  // namespace bpmax
