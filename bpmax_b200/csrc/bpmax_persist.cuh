// bpmax_persist.cuh -- the fill of one width class (Np <= 64, cell images) as ONE persistent kernel
// that walks the outer diagonals as a wavefront with device-side dependency counters.
//
// The graph path (bpmax_engine.cu) runs every outer diagonal as a product launch and a finalize
// launch, so the stream order is the dependency. Here one launch per width class does all of it:
// its CTAs (the product kernel's shape, R0Cfg<NB>) claim work items in a fixed order from a queue
// with an atomic counter and wait, bounded, for each item's dependencies on counters in global
// memory:
//   product job (cell (i1, i1+d), k1 offset pairs [p0, p1), as R0Job): reads the tables of the
//     diagonals w and d-1-w (w in the job's pairs); the finalize of diagonal d-2 also pushes the
//     SW1 candidates into the (cleared) tables of diagonal d, which the product merges into with
//     atomicMax. So the job waits until every cell of diagonal d-1 (p0 == 0) or d-2 (p0 >= 1) is
//     finalized (diag_done[pair][e] == M - e; a diagonal complete implies every earlier one is);
//   finalize of cell (i1, i1+d): waits until all its product jobs have merged (prod_done[cell] ==
//     prod_need[cell]); it computes S1(i1, i1+d) itself from S1 of shorter intervals (final since
//     the cell's offset-pair-0 job waited for diagonal d-1), runs the inner wavefront (R1, R2, SW2)
//     with the CTA's threads, writes the table, its S1 pieces and the SW1 push into the cleared
//     table of (i1-1, i1+d+1), and counts itself in diag_done[pair][d].
// The host orders the queue so that every item depends only on items before it: for d = 1, 2, ...
// the finalize items of diagonal d-1, then the jobs of diagonal d with p0 >= 1 (they run beside
// those finalizes), then the jobs of d with p0 == 0; the finalize items of the last diagonal close
// the queue. Items are claimed in queue order by running CTAs, one item ahead (a CTA claims its next
// item while it works on the current one, and stages the item and its pair's descriptor in shared
// memory, so the claim and those loads are off the critical path). The earliest unfinished claimed
// item always has its dependencies finished, and its CTA has finished everything it claimed before
// it: the schedule makes progress whatever number of CTAs is resident.
// Publishing: every thread fences its writes (__threadfence), the CTA barrier joins them, and one
// thread adds to the counter; the waiting thread reads the counter with ld.acquire.gpu, the CTA
// barrier hands the result on, tables written by other CTAs are read with L2-only loads, and a
// proxy fence orders them before the product's bulk copies (async proxy).
// Waits are bounded: a wait that runs out, or finds the error word set, sets the error word and
// makes the CTA drain its copies in flight (bounded) and leave; every later wait of any CTA then
// fails at once, so a failing fill ends within about one wait limit.
#pragma once
#include "bpmax_r0.cuh"

namespace bpmax {

// one work item of the queue: kind 0 = product job (cell (i1, i1+d), offset pairs [p0, p1)),
// kind 1 = finalize of cell (i1, i1+d)
struct PItem {
    int pair, i1, d, p0, p1, kind;
};

struct PersistCtl {
    const PItem *items;    // this class's queue
    int nitems;
    int *head;             // next item to claim (cleared before the launch)
    int *diag_done;        // [PairDesc::cnt_off + e]: cells of outer diagonal e finalized
    int *prod_done;        // [PairDesc::cell_base + cell]: product jobs of the cell merged
    const int *prod_need;  // [PairDesc::cell_base + cell]: product jobs of the cell
};

__device__ __forceinline__ int ld_acquire(const int *p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// bounded wait (one thread) until *p >= target; false when the limit ran out or the error word is set
__device__ __noinline__ bool wait_count(const int *p, int target, const int *err, unsigned long long limit_ns)
{
    for (int i = 0; i < 32; ++i)
        if (ld_acquire(p) >= target) return true;
    const unsigned long long t0 = globaltimer_ns();
    while (true) {
        if (ld_acquire(p) >= target) return true;
        if (ld_acquire(err) != 0 || globaltimer_ns() - t0 > limit_ns) return false;
        __nanosleep(256);
    }
}

template <int NB>
struct PersistCfg {
    using C = R0Cfg<NB>;
    static constexpr int NP = 8 * NB;
    static constexpr int THREADS = C::THREADS;
    static constexpr int WARPS = THREADS / 32;
    static constexpr int K = (NP * (NP - 1) / 2 + THREADS - 1) / THREADS;  // owned inner cells per thread
    static constexpr int FIN_BYTES = 2 * NP * NP * 4 + NP;                  // D, S2, bases (inside the ring)
    static_assert(FIN_BYTES <= C::OFF_RED, "the finalize's tables fit in the product's stages");
    static_assert(K <= 24, "slots");
    static_assert(THREADS >= 64, "warp 1 claims the next item");
    static_assert(sizeof(PItem) == 24 && sizeof(PairDesc) % 8 == 0 && sizeof(PairDesc) / 8 <= 32, "staged descriptors");
};

template <int NB>
__global__ void __launch_bounds__(R0Cfg<NB>::THREADS, R0Cfg<NB>::MINB)
fill_persistent_kernel(PersistCtl pc, const PairDesc *__restrict__ pairs, float *__restrict__ F, float *__restrict__ S,
                       const uint8_t *__restrict__ bases, Weights W, WaitCtl ctl)
{
    using C = R0Cfg<NB>;
    using P = PersistCfg<NB>;
    constexpr int SS = C::STAGES, NP = P::NP, NBLK = C::NBLK, K = P::K;
    constexpr long long CELL = 4LL * C::IMG;
    extern __shared__ __align__(128) float psm[];
    int *red = reinterpret_cast<int *>(reinterpret_cast<char *>(psm) + C::OFF_RED);
    int *red_dst = reinterpret_cast<int *>(reinterpret_cast<char *>(psm) + C::OFF_DST);
    uint64_t *bars = reinterpret_cast<uint64_t *>(reinterpret_cast<char *>(psm) + C::OFF_BAR);
    int *done_cnt = reinterpret_cast<int *>(reinterpret_cast<char *>(psm) + C::OFF_CNT);
    int *armed = reinterpret_cast<int *>(reinterpret_cast<char *>(psm) + C::OFF_ARM);
    __shared__ int ok_sh;
    __shared__ int idx_sh[2];                             // claimed items, double-buffered
    __shared__ int itm_sh[2][6];                          // their PItem
    __shared__ long long pd_sh[2][sizeof(PairDesc) / 8];  // and their pair's descriptor
    __shared__ float s1_sh;
    __shared__ float wsh[12];
    __shared__ int cbs[NB];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        for (int s = 0; s < SS; ++s) {
            mbar_init(smem_u32(bars + s), 1);
            done_cnt[s] = 0;
            armed[s] = 0;
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int q = tid; q < C::RED_WORDS; q += C::THREADS) red[q] = 0;
    if (tid < NBLK) {
        int bi_ = 0, bj_ = tid;
        while (bj_ >= NB - bi_) { bj_ -= NB - bi_; ++bi_; }
        bj_ += bi_;
        red_dst[tid] = 4 * (c_img_colbase[NB][bj_] + 17 * bi_);
    }
    if (tid < 12) wsh[tid] = W.w[tid];
    if (tid < NB) cbs[tid] = 4 * c_img_colbase[NB][tid];

    // the lane's product task (as r0_kernel)
    const int role = (int)(C::ROLE_BITS >> (2 * (tid >> 5))) & 3;
    const unsigned char *lt = c_r0_lane[NB - 1][tid];
    const bool has_task = lt[0] != 255;
    const int tg = has_task ? lt[0] : 0, bi = lt[1], bj = lt[2], kb = lt[3];
    int a_off = 0, b_off = 0, r3_off = 0, red_off = 0;
    if (has_task) {
        red_off = 65 * (bi * NB - bi * (bi - 1) / 2 + (bj - bi));
        a_off = 4 * (c_img_colbase[NB][kb] + 17 * bi);
        b_off = 4 * (C::IMG + c_img_colbase[NB][bj] + 17 * kb + 2);
        r3_off = 4 * (C::IMG + c_img_colbase[NB][bj] + 17 * bi);
    }
    const unsigned smem_base = smem_u32(psm);
    unsigned phase = 0;  // bit s: parity of stage s's next completion (kept across jobs)
    // one full warp claims the next item and stages it and its pair's descriptor in slot t
    auto claim = [&](int t) {
        int nx = 0;
        if (lane == 0) nx = atomicAdd(pc.head, 1);
        nx = __shfl_sync(0xffffffffu, nx, 0);
        if (lane == 0) idx_sh[t] = nx;
        if (nx < pc.nitems) {
            const int w = lane < 6 ? reinterpret_cast<const int *>(pc.items + nx)[lane] : 0;
            if (lane < 6) itm_sh[t][lane] = w;
            const int pr = __shfl_sync(0xffffffffu, w, 0);  // PItem::pair
            if (lane < (int)(sizeof(PairDesc) / 8)) pd_sh[t][lane] = reinterpret_cast<const long long *>(pairs + pr)[lane];
        }
    };
    if (warp == 0) claim(0);
    __syncthreads();

#pragma unroll 1
    for (int t = 0;; t ^= 1) {  // slot t holds the current item; the next one is claimed into t ^ 1
        const int idx = idx_sh[t];
        if (idx >= pc.nitems) break;
        const PItem itm = *reinterpret_cast<const PItem *>(itm_sh[t]);
        const PairDesc pd = *reinterpret_cast<const PairDesc *>(pd_sh[t]);
        const int M = pd.M, d = itm.d, i1 = itm.i1, j1 = i1 + d;
        const long long cell = pd.cell_base + cell_index(M, i1, j1);
        // dependency wait (thread 0), its result to every thread
        if (tid == 0) {
            bool ok;
            if (itm.kind == 0) {
                const int dep = itm.p0 == 0 ? d - 1 : d - 2;
                ok = dep < 0 || wait_count(pc.diag_done + pd.cnt_off + dep, M - dep, ctl.err, ctl.wait_ns);
            } else {
                ok = wait_count(pc.prod_done + cell, pc.prod_need[cell], ctl.err, ctl.wait_ns);
            }
            if (!ok) atomicExch(ctl.err, 1);
            ok_sh = ok;
        }
        __syncthreads();
        if (!ok_sh) break;

        if (itm.kind == 0) {
            // ---------------------------------------------------------------- product job
            // tables of other CTAs (global) and this CTA's finalize tables in the ring (shared), both
            // written through the generic proxy, before the bulk copies (async proxy)
            asm volatile("fence.proxy.async.global;\n\tfence.proxy.async.shared::cta;" ::: "memory");
            const R0Job job{itm.pair, i1, itm.p0, itm.p1};
            const int items = r0_job_items(job, d), iters = (items + C::G - 1) / C::G;
            const float *Fp = F + pd.F_off;
            auto expect = [&](int s, int it_) {
                const int valid = min(C::G, items - it_ * C::G);
                mbar_arrive_tx(smem_u32(bars + s), (unsigned)(valid * C::ITEM_TX));
                armed[s] += 1;
            };
            auto issue = [&](int s, int it_, int me, int count) {
                const int valid = min(C::G, items - it_ * C::G);
                const unsigned bar = smem_u32(bars + s);
                for (int o = me; o < 2 * valid; o += count) {
                    const int g = o >> 1, k1 = i1 + r0_item_offset(job, d, it_ * C::G + g);
                    const long long cl = (o & 1) ? cell_index(M, k1 + 1, j1) : cell_index(M, i1, k1);
                    bulk_g2s(smem_base + (unsigned)(s * C::STAGE_BYTES + (g * C::ITEM + (o & 1) * C::IMG) * 16),
                             Fp + cl * CELL, (unsigned)(C::IMG * 16), bar);
                }
            };
            const int prime = min(SS, iters);
            if (tid == 0 && !ctl.inject)
                for (int s = 0; s < prime; ++s) expect(s, s);
            __syncthreads();
            if (!ctl.inject)
                for (int s = 0; s < prime; ++s) issue(s, s, tid, C::THREADS);
            if (warp == 1) claim(t ^ 1);
            float acc[8][8];
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] = NEG_INF;
            bool bad = false;
#pragma unroll 1
            for (int it = 0; it < iters; ++it) {
                const int stage = it % SS;
                const bool active = has_task && it * C::G + tg < items;
                if (!bad && !mbar_wait(smem_u32(bars + stage), (phase >> stage) & 1u, ctl.wait_ns)) {
                    atomicExch(ctl.err, 1);
                    bad = true;
                }
                phase ^= 1u << stage;
                if (active && !bad) {
                    const float *item = psm + (size_t)stage * C::STAGE * 4 + tg * C::ITEM * 4;
                    const float *As = item + a_off, *Bs = item + b_off;
                    if (role == 0)
                        r0_task<0>(As, Bs, acc);
                    else if (role == 1)
                        r0_task<1>(As, Bs, acc);
                    else if (role == 2)
                        r0_task<2>(As, Bs, acc);
                    else
                        r0_task<3>(As, Bs, acc);
                    if (kb == bi) {
                        const float s1a = item[8];
                        const float4 r0 = *reinterpret_cast<const float4 *>(item + r3_off);
                        const float4 r1 = *reinterpret_cast<const float4 *>(item + r3_off + 4);
                        const float rv[8] = {r0.x, r0.y, r0.z, r0.w, r1.x, r1.y, r1.z, r1.w};
#pragma unroll
                        for (int j = 0; j < 8; ++j) acc[0][j] = fmaxf(acc[0][j], s1a + rv[j]);
                    }
                }
                __syncwarp();
                int last = 0;
                if (lane == 0) last = atomicAdd(done_cnt + stage, 1) == C::WARPS - 1;
                last = __shfl_sync(0xffffffffu, last, 0);
                if (last && it + SS < iters && !__any_sync(0xffffffffu, bad)) {
                    if (lane == 0) {
                        done_cnt[stage] = 0;
                        expect(stage, it + SS);
                    }
                    __syncwarp();
                    issue(stage, it + SS, lane, 32);
                } else if (last && lane == 0) {
                    done_cnt[stage] = 0;
                }
            }
            // merge the partial maxima into F(i1, j1), then count the job
            if (has_task) {
#pragma unroll
                for (int i = 0; i < 8; ++i)
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const int i2 = 8 * bi + i, j2 = 8 * bj + j;
                        const int v = __float_as_int(acc[i][j]);
                        if (i2 <= j2 && j2 < pd.N && v > 0) atomicMax(red + red_off + 8 * i + j, v);
                    }
            }
            if (__syncthreads_or(bad)) {
                if (tid == 0) mbar_drain(bars, armed, SS, ctl.wait_ns);
                break;
            }
            int *out = reinterpret_cast<int *>(F + pd.F_off + cell_index(M, i1, j1) * CELL);
            for (int e = tid; e < 64 * NBLK; e += C::THREADS) {
                const int q = e >> 6, w = e & 63;
                const int v = red[65 * q + w];
                if (v > 0) {
                    atomicMax(out + red_dst[q] + w, v);
                    red[65 * q + w] = 0;
                }
            }
            __threadfence();
            __syncthreads();
            if (tid == 0) atomicAdd(pc.prod_done + cell, 1);
            continue;
        }

        // -------------------------------------------------------------------- finalize of the cell
        // (the inner wavefront of finalize_small_kernel with this CTA's threads; its tables live in
        // the stages of the product ring, idle between jobs)
        const int N = pd.N;
        float *Fc = F + pd.F_off + cell_index(M, i1, j1) * CELL;
        float *S1g = S + pd.S1_off;
        const float *S2g = S + pd.S2_off;
        const uint8_t *s1 = bases + pd.seq1_off;
        const uint8_t *s2r = bases + pd.seq2_off;
        float *D = psm, *S2s = psm + NP * NP;
        uint8_t *sb = reinterpret_cast<uint8_t *>(psm + 2 * NP * NP);
        if (warp == 1) claim(t ^ 1);
        if (warp == 0) {  // S1(i1, j1) from the final S1 of shorter intervals (0 while j1 - i1 <= 3)
            float v = 0.0f;
            if (d > 3) {
                float red1 = NEG_INF;
                for (int k = i1 + lane; k < j1; k += 32) red1 = fmaxf(red1, __ldcg(S1g + i1 * M + k) + __ldcg(S1g + (k + 1) * M + j1));
                for (int o = 16; o > 0; o >>= 1) red1 = fmaxf(red1, __shfl_xor_sync(0xffffffffu, red1, o));
                v = fmaxf(__ldcg(S1g + (i1 + 1) * M + (j1 - 1)) + score_w(wsh, s1[i1], s1[j1]), red1);
                if (lane == 0) S1g[i1 * M + j1] = v;
            }
            if (lane == 0) s1_sh = v;
        }
        for (int q4 = tid; q4 < NP * NP / 4; q4 += C::THREADS)
            *reinterpret_cast<float4 *>(S2s + 4 * q4) = *reinterpret_cast<const float4 *>(S2g + 4 * q4);
        for (int q = tid; q < NP; q += C::THREADS) sb[q] = q < N ? s2r[q] : 4;
        __syncthreads();
        const float s1v = s1_sh;
        auto img = [&](int r, int c) { return __ldcg(Fc + cbs[c >> 3] + 68 * (r >> 3) + 8 * (r & 7) + (c & 7)); };
        const int ncells = N * (N - 1) / 2;
        int cell_i[K], cell_e[K];
        float facc[K], sw2[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int c = tid + C::THREADS * k;
            cell_e[k] = NP;
            cell_i[k] = 0;
            facc[k] = NEG_INF;
            sw2[k] = NEG_INF;
            if (c < ncells) {
                int e = 1, rem = c;
                while (rem >= N - e) { rem -= N - e; ++e; }
                cell_e[k] = e;
                cell_i[k] = rem;
                facc[k] = fmaxf(img(rem, rem + e), s1v + S2s[rem * NP + rem + e]);
                if (e >= 4) sw2[k] = score_w(wsh, sb[rem], sb[rem + e]);
            }
        }
        if (tid < N) D[tid] = d == 0 ? score_w(wsh + 6, s1[i1], sb[tid]) : fmaxf(img(tid, tid), s1v + S2s[tid * NP + tid]);
        __syncthreads();
        for (int e = 0; e + 1 < N; ++e) {
            const float *De = D + e * NP;
            const int first = (e * N - e * (e + 1) / 2) / C::THREADS;  // slots before it hold final cells only
#pragma unroll
            for (int k = 0; k < K; ++k) {
                if (k < first) continue;  // uniform over the CTA
                const int e2 = cell_e[k];
                if (e2 > e && e2 < NP) {
                    const int i2 = cell_i[k], j2 = i2 + e2;
                    facc[k] = fmax3(facc[k], De[i2] + S2s[(i2 + e + 1) * NP + j2], S2s[i2 * NP + j2 - e - 1] + De[j2 - e]);
                    if (e2 == e + 1) D[e2 * NP + i2] = fmaxf(facc[k], D[max(e2 - 2, 0) * NP + i2 + 1] + sw2[k]);
                }
            }
            __syncthreads();
        }
        const bool push = i1 >= 1 && j1 + 1 < M && d + 2 >= 4;
        const float wp = push ? score_w(wsh, s1[i1 - 1], s1[j1 + 1]) : 0.0f;
        float *Fn = push ? F + pd.F_off + cell_index(M, i1 - 1, j1 + 1) * CELL : nullptr;
        for (int q4 = tid; q4 < NBLK * 16; q4 += C::THREADS) {
            int BI, BJ;
            blk_decode(NB, q4 >> 4, BI, BJ);
            const int r = 8 * BI + ((q4 & 15) >> 1), c0 = 8 * BJ + 4 * (q4 & 1);
            float v[4], u[4];
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                const int c = c0 + t;
                const bool valid = r <= c && c < N;
                v[t] = valid ? D[(c - r) * NP + r] : (r == c + 1 ? s1v : NEG_INF);
                u[t] = valid ? v[t] + wp : 0.0f;
            }
            const int o = cbs[BJ] + 68 * BI + 4 * (q4 & 15);
            if (push) *reinterpret_cast<float4 *>(Fn + o) = make_float4(u[0], u[1], u[2], u[3]);
            *reinterpret_cast<float4 *>(Fc + o) = make_float4(v[0], v[1], v[2], v[3]);
        }
        if (tid < 2 * NB) {
            const int BJ = tid >> 1, h = tid & 1;
            float4 p4 = make_float4(NEG_INF, NEG_INF, NEG_INF, NEG_INF);
            if (h == 1) p4.w = s1v;
            *reinterpret_cast<float4 *>(Fc + cbs[BJ] + 68 * (BJ + 1) + 4 * h) = p4;
        }
        __threadfence();
        __syncthreads();
        if (tid == 0) atomicAdd(pc.diag_done + pd.cnt_off + d, 1);
    }
}

}  // namespace bpmax
