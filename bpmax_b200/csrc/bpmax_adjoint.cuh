// bpmax_adjoint.cuh -- adjoint (backward) pass of the BPMax fill: d score / d weights.
//
// The optimal score is a max over structures; its derivative with respect to weight t is the
// number of times the optimal structure uses pair type t. The adjoint of the root is 1 and every
// max passes it to its winning candidate only, so the derivative follows the argmax edges from
// F(0,M-1,0,N-1) down to the leaves, adding 1 to a weight's count at every scored pair.
// No back-pointers are stored: each visited node recomputes its candidates from the stored F, S1
// and S2 (every candidate is one fp32 add of two stored values, so the recomputed values are
// the forward values bit for bit) and picks the winner with the tie-break of the reference's
// right-nested __max_float(x,y) = x>y ? x : y (V3/bpmax_verify.c, eval_FTable :576):
//   * among the node's candidates, in the order SW1, SW2, S1+S2, R0, R1, R2, R3, R4 (a literal 0
//     where a term is undefined), the LAST one attaining the maximum wins;
//   * inside a reduction (reduceVar = __max_float(reduceVar, temp), :586) the LAST k attaining the
//     maximum wins, k1 outer and k2 inner for R0 (:591-597).
// Both rules are one 64-bit max over (value bits << 32 | position): values are >= +0, so their
// bit patterns order like the floats.
#pragma once
#include "bpmax_kernels.cuh"

namespace bpmax {

enum { TB_F = 0, TB_S1 = 1, TB_S2 = 2 };
struct TbNode {
    int kind, a, b, c;  // F: a = i1<<16|j1, b = i2<<16|j2 ; S1/S2: a = i, b = j
};

__device__ __forceinline__ unsigned long long tb_key(float v, unsigned idx)
{
    return ((unsigned long long)__float_as_uint(v) << 32) | idx;
}

template <int NT>
__device__ __forceinline__ void tb_block_max(unsigned long long (&k)[5], unsigned long long (*sh)[5])
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int g = 0; g < 5; ++g)
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long x = __shfl_xor_sync(0xffffffffu, k[g], o);
            k[g] = x > k[g] ? x : k[g];
        }
    if (lane == 0)
#pragma unroll
        for (int g = 0; g < 5; ++g) sh[warp][g] = k[g];
    __syncthreads();
    if (threadIdx.x == 0)
        for (int w = 1; w < NT / 32; ++w)
#pragma unroll
            for (int g = 0; g < 5; ++g) sh[0][g] = sh[w][g] > sh[0][g] ? sh[w][g] : sh[0][g];
    __syncthreads();
}

constexpr int TB_THREADS = 256;

// One CTA per pair. stacks: cap nodes per pair. grads: 12 per pair. status[pair] = 0 ok,
// 1 stack overflow, 2 node budget exhausted (both bounded: the kernel always returns).
__global__ void __launch_bounds__(TB_THREADS)
traceback_kernel(const PairDesc *__restrict__ pairs, const float *__restrict__ F, const float *__restrict__ S,
                 const uint8_t *__restrict__ bases, Weights W, TbNode *__restrict__ stacks, int cap,
                 float *__restrict__ grads, int *__restrict__ status)
{
    const PairDesc pd = pairs[blockIdx.x];
    const int M = pd.M, N = pd.N, Np = pd.Np;
    const float *S1 = S + pd.S1_off;
    const float *S2 = S + pd.S2_off;
    const uint8_t *s1 = bases + pd.seq1_off;
    const uint8_t *s2r = bases + pd.seq2_off;
    TbNode *st = stacks + (long long)blockIdx.x * cap;
    __shared__ int sp, done, err;
    __shared__ TbNode cur;
    __shared__ float cnt[12];
    __shared__ unsigned long long red[TB_THREADS / 32][5];
    auto Fv = [&](int a, int b, int x, int y) { return f_value(pd, F, cell_index(M, a, b), x, y); };
    const int tid = threadIdx.x;
    if (tid < 12) cnt[tid] = 0.0f;
    if (tid == 0) {
        sp = 1;
        err = 0;
        st[0] = TbNode{TB_F, (0 << 16) | (M - 1), (0 << 16) | (N - 1), 0};
    }
    __syncthreads();
    const long long budget = 64LL * (M + N) + 4096;
    for (long long it = 0;; ++it) {
        if (tid == 0) {
            done = sp == 0 || err != 0;
            if (!done && it >= budget) { err = 2; done = 1; }
            if (!done) cur = st[--sp];
        }
        __syncthreads();
        if (done) break;
        const TbNode n = cur;
        unsigned long long k[5] = {0, 0, 0, 0, 0};
        if (n.kind != TB_F) {
            const bool two = n.kind == TB_S2;
            const int i = n.a, j = n.b, L = two ? Np : M;
            const float *T = two ? S2 : S1;
            const uint8_t *s = two ? s2r : s1;
            if (j - i <= 3) { __syncthreads(); continue; }  // literal 0: no pair
            for (int q = tid; q < j - i; q += TB_THREADS) {
                const int kk = i + q;
                const unsigned long long x = tb_key(T[i * L + kk] + T[(kk + 1) * L + j], q);
                k[0] = x > k[0] ? x : k[0];
            }
            tb_block_max<TB_THREADS>(k, red);
            if (tid == 0) {
                const float pr = T[(i + 1) * L + (j - 1)] + score_w(W.w, s[i], s[j]);
                const float rv = __uint_as_float((unsigned)(red[0][0] >> 32));
                const int rk = i + (int)(red[0][0] & 0xffffffffu);
                if (sp + 2 > cap) err = 1;
                else if (pr > rv) {  // __max_float(pair, reduction): the pair wins only when strictly larger
                    const int t = pair_type(s[i], s[j]);
                    if (t >= 0) cnt[t] += 1.0f;
                    st[sp++] = TbNode{n.kind, i + 1, j - 1, 0};
                } else {
                    st[sp++] = TbNode{n.kind, i, rk, 0};
                    st[sp++] = TbNode{n.kind, rk + 1, j, 0};
                }
            }
            __syncthreads();
            continue;
        }
        const int i1 = n.a >> 16, j1 = n.a & 0xffff, i2 = n.b >> 16, j2 = n.b & 0xffff;
        const int d1 = j1 - i1, d2 = j2 - i2;
        if (d1 == 0 && d2 == 0) {  // base case: one inter-strand pair
            if (tid == 0) {
                const int t = pair_type(s1[i1], s2r[i2]);
                if (t >= 0) cnt[6 + t] += 1.0f;
            }
            __syncthreads();
            continue;
        }
        // candidate groups R0..R4 evaluated in parallel over one flat index space
        const int n0 = (d1 >= 1 && d2 >= 1) ? d1 * d2 : 0, n12 = d2 >= 1 ? d2 : 0, n34 = d1 >= 1 ? d1 : 0;
        const int total = n0 + 2 * n12 + 2 * n34;
        for (int q = tid; q < total; q += TB_THREADS) {
            int g, idx;
            float v;
            if (q < n0) {
                g = 0;
                idx = q;
                const int k1 = i1 + q / d2, k2 = i2 + q % d2;
                v = Fv(i1, k1, i2, k2) + Fv(k1 + 1, j1, k2 + 1, j2);
            } else if (q < n0 + n12) {
                g = 1;
                idx = q - n0;
                const int k2 = i2 + idx;
                v = Fv(i1, j1, i2, k2) + S2[(k2 + 1) * Np + j2];
            } else if (q < n0 + 2 * n12) {
                g = 2;
                idx = q - n0 - n12;
                const int k2 = i2 + idx;
                v = S2[i2 * Np + k2] + Fv(i1, j1, k2 + 1, j2);
            } else if (q < n0 + 2 * n12 + n34) {
                g = 3;
                idx = q - n0 - 2 * n12;
                const int k1 = i1 + idx;
                v = S1[i1 * M + k1] + Fv(k1 + 1, j1, i2, j2);
            } else {
                g = 4;
                idx = q - n0 - 2 * n12 - n34;
                const int k1 = i1 + idx;
                v = Fv(i1, k1, i2, j2) + S1[(k1 + 1) * M + j1];
            }
            const unsigned long long x = tb_key(v, (unsigned)idx);
            k[g] = x > k[g] ? x : k[g];
        }
        tb_block_max<TB_THREADS>(k, red);
        if (tid == 0) {
            // candidates in the order of eval_FTable; tag: 0 SW1 1 SW2 2 S1+S2 3..7 R0..R4, 8 literal 0
            float val[8];
            int tag[8];
            val[0] = d1 >= 4 ? Fv(i1 + 1, j1 - 1, i2, j2) + score_w(W.w, s1[i1], s1[j1]) : 0.0f;
            tag[0] = d1 >= 4 ? 0 : 8;
            val[1] = d2 >= 4 ? Fv(i1, j1, i2 + 1, j2 - 1) + score_w(W.w, s2r[i2], s2r[j2]) : 0.0f;
            tag[1] = d2 >= 4 ? 1 : 8;
            val[2] = S1[i1 * M + j1] + S2[i2 * Np + j2];
            tag[2] = 2;
            const bool has[5] = {n0 > 0, n12 > 0, n12 > 0, n34 > 0, n34 > 0};
            for (int g = 0; g < 5; ++g) {
                val[3 + g] = has[g] ? __uint_as_float((unsigned)(red[0][g] >> 32)) : 0.0f;
                tag[3 + g] = has[g] ? 3 + g : 8;
            }
            int w = 0;
            for (int c = 1; c < 8; ++c)
                if (!(val[w] > val[c])) w = c;  // right-nested __max_float: the last maximum wins
            const int widx = tag[w] >= 3 && tag[w] <= 7 ? (int)(red[0][tag[w] - 3] & 0xffffffffu) : 0;
            if (sp + 2 > cap) err = 1;
            else switch (tag[w]) {
                case 0: {
                    const int t = pair_type(s1[i1], s1[j1]);
                    if (t >= 0) cnt[t] += 1.0f;
                    st[sp++] = TbNode{TB_F, ((i1 + 1) << 16) | (j1 - 1), n.b, 0};
                } break;
                case 1: {
                    const int t = pair_type(s2r[i2], s2r[j2]);
                    if (t >= 0) cnt[t] += 1.0f;
                    st[sp++] = TbNode{TB_F, n.a, ((i2 + 1) << 16) | (j2 - 1), 0};
                } break;
                case 2:
                    st[sp++] = TbNode{TB_S1, i1, j1, 0};
                    st[sp++] = TbNode{TB_S2, i2, j2, 0};
                    break;
                case 3: {
                    const int k1 = i1 + widx / d2, k2 = i2 + widx % d2;
                    st[sp++] = TbNode{TB_F, (i1 << 16) | k1, (i2 << 16) | k2, 0};
                    st[sp++] = TbNode{TB_F, ((k1 + 1) << 16) | j1, ((k2 + 1) << 16) | j2, 0};
                } break;
                case 4: {
                    const int k2 = i2 + widx;
                    st[sp++] = TbNode{TB_F, n.a, (i2 << 16) | k2, 0};
                    st[sp++] = TbNode{TB_S2, k2 + 1, j2, 0};
                } break;
                case 5: {
                    const int k2 = i2 + widx;
                    st[sp++] = TbNode{TB_S2, i2, k2, 0};
                    st[sp++] = TbNode{TB_F, n.a, ((k2 + 1) << 16) | j2, 0};
                } break;
                case 6: {
                    const int k1 = i1 + widx;
                    st[sp++] = TbNode{TB_S1, i1, k1, 0};
                    st[sp++] = TbNode{TB_F, ((k1 + 1) << 16) | j1, n.b, 0};
                } break;
                case 7: {
                    const int k1 = i1 + widx;
                    st[sp++] = TbNode{TB_F, (i1 << 16) | k1, n.b, 0};
                    st[sp++] = TbNode{TB_S1, k1 + 1, j1, 0};
                } break;
                default: break;  // literal 0: empty structure
                }
        }
        __syncthreads();
    }
    if (tid < 12) grads[blockIdx.x * 12 + tid] = cnt[tid];
    if (tid == 0) status[blockIdx.x] = err;
}

}  // namespace bpmax
