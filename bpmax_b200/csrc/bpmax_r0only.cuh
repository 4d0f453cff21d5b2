// bpmax_r0only.cuh -- the R0-only double max-plus microbenchmark on the fill's own product
// kernels. It restates the reference's IPDPSW R0-only program
// (IPDPSW/source/R0/ospsq_coarse_diag_top_down/ospsq_float.ab:1-15, kernel
// IPDPSW/source/R0/ospsq_coarse_diag_top_down/src/ospsqmax_float.c:113-189):
//   F(i1,i1,i2,j2) = seq2[i2]
//   F(i1,j1,i2,i2) = seq1[i1]                                                  (j1 > i1)
//   F(i1,j1,i2,j2) = max_{i1<=k1<j1, i2<=k2<j2} F(i1,k1,i2,k2) + F(k1+1,j1,k2+1,j2)   (j1 > i1, j2 > i2)
// The product kernels evaluate R0 + R3 + R4 as one shifted product whose extra terms read S1 on the
// subdiagonal of every table (and, for wide tables, the S1 array): with -inf there, they evaluate
// R0 alone. The finalize of this mode only writes the base values and -inf where the full fill
// writes S1; the sequences are non-negative, so every value is >= +0 and the product's integer
// max merge stays exact.
#pragma once
#include "bpmax_kernels_large.cuh"

namespace bpmax {

// S1 := -inf for every pair (read by the wide product kernel at row 0 of A and the guard row of B)
__global__ void r0only_prep_kernel(const PairDesc *__restrict__ pairs, float *__restrict__ S)
{
    const PairDesc pd = pairs[blockIdx.x];
    float *S1 = S + pd.S1_off;
    for (int q = threadIdx.x; q < pd.M * pd.M; q += blockDim.x) S1[q] = NEG_INF;
}

// Cell images (Np <= 64), one CTA per outer cell of diagonal d. vals = seq1 (M floats) then seq2
// (N floats) of the pair, unreversed.
template <int NP>
__global__ void __launch_bounds__(128) r0only_finalize_small_kernel(const CellJob *__restrict__ jobs,
                                                                   const PairDesc *__restrict__ pairs,
                                                                   float *__restrict__ F,
                                                                   const float *__restrict__ vals, int d)
{
    constexpr int NB = NP / 8, NBLK = NB * (NB + 1) / 2;
    constexpr long long CELL = 4LL * R0_TAB_COLBASE[NB][NB];
    const CellJob job = jobs[blockIdx.x];
    const PairDesc pd = pairs[job.pair];
    const int M = pd.M, N = pd.N, i1 = job.i1;
    float *Fc = F + pd.F_off + cell_index(M, i1, i1 + d) * CELL;
    const float *v1 = vals, *v2 = vals + M;
    for (int q4 = threadIdx.x; q4 < NBLK * 16; q4 += blockDim.x) {
        int BI, BJ;
        blk_decode(NB, q4 >> 4, BI, BJ);
        const int r = 8 * BI + ((q4 & 15) >> 1), c0 = 8 * BJ + 4 * (q4 & 1);
        const int o = 4 * c_img_colbase[NB][BJ] + 68 * BI + 4 * (q4 & 15);  // block (BI, BJ), row r & 7, half
        const float4 acc = *reinterpret_cast<const float4 *>(Fc + o);
        const float a[4] = {acc.x, acc.y, acc.z, acc.w};
        float v[4];
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            const int c = c0 + t;
            v[t] = !(r <= c && c < N) ? NEG_INF : (d == 0 ? v2[r] : (r == c ? v1[i1] : a[t]));
        }
        *reinterpret_cast<float4 *>(Fc + o) = make_float4(v[0], v[1], v[2], v[3]);
    }
    if (threadIdx.x < 2 * NB) {  // S1 piece of every block column: all -inf here
        const int BJ = threadIdx.x >> 1, h = threadIdx.x & 1;
        *reinterpret_cast<float4 *>(Fc + 4 * c_img_colbase[NB][BJ] + 68 * (BJ + 1) + 4 * h) =
            make_float4(NEG_INF, NEG_INF, NEG_INF, NEG_INF);
    }
}

// Tile images (64 < Np <= WIDE_TILE_MAX_NP): one CTA per outer cell of diagonal d rewrites every
// block of every tile with the base values and -inf where the full fill writes S1, and writes the
// closing pieces (S1 pieces of the diagonal tiles: -inf; halo pieces of the dense tiles: the row
// after the tile, by the same rule). The rule is idempotent, so reading an entry another thread
// has already rewritten gives the same value.
__global__ void __launch_bounds__(256) r0only_finalize_tile_kernel(const CellJob *__restrict__ jobs,
                                                                  const PairDesc *__restrict__ pairs,
                                                                  float *__restrict__ F,
                                                                  const float *__restrict__ vals, int d)
{
    const CellJob job = jobs[blockIdx.x];
    const PairDesc pd = pairs[job.pair];
    const int M = pd.M, N = pd.N, NT = pd.Np >> 6, i1 = job.i1;
    float *Fc = F + pd.F_off + cell_index(M, i1, i1 + d) * wide_cell_floats(NT);
    const float *v1 = vals, *v2 = vals + M;
    auto val = [&](int r, int c) {
        return !(r <= c && c < N) ? NEG_INF : (d == 0 ? v2[r] : (r == c ? v1[i1] : Fc[wide_pos(NT, r, c)]));
    };
    for (int I = 0; I < NT; ++I)
        for (int J = I; J < NT; ++J) {
            const long long to = wide_tile_off(NT, I, J);
            const int nblk = I == J ? 36 : 64;
            for (int q4 = threadIdx.x; q4 < nblk * 16 + 16; q4 += blockDim.x) {
                if (q4 >= nblk * 16) {
                    const int bj = (q4 - nblk * 16) >> 1, h = q4 & 1;
                    float v[4];
#pragma unroll
                    for (int t = 0; t < 4; ++t) v[t] = I == J ? NEG_INF : val(64 * I + 64, 64 * J + 8 * bj + 4 * h + t);
                    const int cb = I == J ? c_img_colbase[8][bj] : c_wide_dense_colbase[bj];
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
                float v[4];
#pragma unroll
                for (int t = 0; t < 4; ++t) v[t] = val(r, c0 + t);
                const long long o = to + 4 * ((I == J ? c_img_colbase[8][bj] : c_wide_dense_colbase[bj]) + 17 * bi) +
                                    4 * (q4 & 15);
                *reinterpret_cast<float4 *>(Fc + o) = make_float4(v[0], v[1], v[2], v[3]);
            }
        }
}

// Row-major tables and their transposes (Np > WIDE_TILE_MAX_NP): CTA (blockIdx.x, blockIdx.y) writes the 32-row
// band blockIdx.y of cell blockIdx.x of diagonal d, one 32 x 32 tile at a time, and the matching
// column band of the transpose through a shared tile (coalesced reads and writes on both sides).
constexpr int R0ONLY_TILE = 32;
__global__ void __launch_bounds__(256) r0only_finalize_wide_kernel(const CellJob *__restrict__ jobs,
                                                                  const PairDesc *__restrict__ pairs,
                                                                  float *__restrict__ F, float *__restrict__ FT,
                                                                  const float *__restrict__ vals, int d)
{
    constexpr int TL = R0ONLY_TILE;
    __shared__ float tile[TL][TL + 1];
    const CellJob job = jobs[blockIdx.x];
    const PairDesc pd = pairs[job.pair];
    const int M = pd.M, N = pd.N, Np = pd.Np, i1 = job.i1;
    const long long cell = cell_index(M, i1, i1 + d) * ((long long)Np * Np);
    float *Fc = F + pd.F_off + cell;
    float *FTc = FT + pd.F_off + cell;
    const float *v1 = vals, *v2 = vals + M;
    const int tx = threadIdx.x & (TL - 1), ty = threadIdx.x / TL;  // 32 x 8 threads
    const int r0 = TL * blockIdx.y;
    for (int c0 = 0; c0 < Np; c0 += TL) {
#pragma unroll
        for (int y = ty; y < TL; y += 8) {
            const int r = r0 + y, c = c0 + tx;
            const long long q = (long long)r * Np + c;
            const float f = !(r <= c && c < N) ? NEG_INF : (d == 0 ? v2[r] : (r == c ? v1[i1] : Fc[q]));
            Fc[q] = f;
            tile[y][tx] = f;
        }
        __syncthreads();
#pragma unroll
        for (int y = ty; y < TL; y += 8)  // FT[c0 + y][r0 + tx] = F[r0 + tx][c0 + y]
            FTc[(long long)(c0 + y) * Np + r0 + tx] = tile[tx][y];
        __syncthreads();
    }
}

}  // namespace bpmax
