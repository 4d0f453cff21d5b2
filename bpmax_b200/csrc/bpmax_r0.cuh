// bpmax_r0.cuh -- R0 + R3 + R4 product kernel for inner tables of width Np = 8*NB <= 64.
//
// For one outer cell (i1, j1 = i1+d) and one k1 in [i1, j1) (an "item"), with A = F(i1,k1) and
// B = F(k1+1,j1) (tables whose subdiagonal holds S1 of their own cell):
//   R0 (V3/bpmax_verify.c:584-613):  max_{k2 in [i2, j2)} A[i2][k2] + B[k2+1][j2]
//   R3 (:668-694):                    S1(i1,k1) + B[i2][j2]      = A[i2][i2-1] + B[i2][j2]
//   R4 (:695-721):                    A[i2][j2] + S1(k1+1,j1)    = A[i2][j2]   + B[j2+1][j2]
// With the row-shifted operand Bs[k][j] = B[k+1][j] all three are one triangular (max,+) product
//   max_{k in [i2-1, j2]} A[i2][k] + Bs[k][j2]
// (every other k meets a -inf below a diagonal). It is split into tasks (bi, bj, kb),
// bi <= kb <= bj: the 8x8 output micro-tile (bi, bj) times the k block [8kb, 8kb+8); a task with
// kb == bi also adds the k = 8bi-1 term of its first row (S1(i1,k1) + B[8bi][j2]), which lies
// outside every k block of the micro-tile.
//
// Data movement: the stored inner table of a cell is a "cell image" (bpmax_kernels.cuh): block
// columns of 8x8 blocks at a pitch of 17 16-byte chunks, each column closed by its S1 piece. An
// item needs exactly two whole images in shared memory, A = F(i1,k1) and B = F(k1+1,j1): two bulk
// copies on the TMA engine (cp.async.bulk, completion counted on the stage's mbarrier). In the
// images, A block (bi,kb) is column kb, block bi; the shifted B block (kb,bj) is rows 1..7 of
// block kb of column bj followed by row 0 of block kb+1 (or, for kb == bj, the column's S1 piece,
// which is exactly row 8kb+8 of B below the block diagonal and, in the last column, the guard row
// B[Np]); the R3 row B[8bi] is row 0 of block bi of column bj. The column pads and the lane ->
// task table (r0_tables.inc) make every quarter-warp's 128-bit loads hit distinct bank groups.
// Stages form a ring without CTA barriers: each warp counts itself done with a stage (shared
// atomic) and the last one refills it with the iteration S ahead.
// Both operands are whole images of the same F tables, so the two uses of a table on one
// diagonal (as A of cell (a, a+d) and as B of cell (b-d, b)) can meet in L2: jobs visit k1
// offsets in pairs (w, d-1-w), the offset pair p = min(w, d-1-w) being the same for both uses,
// and the job list is ordered by offset pair.
//
// The inner loop takes 4 k per step: the 4 rows of the shifted B block in registers, then one A
// row at a time (its 4 operands live only for that row's 32 candidates, which keeps the kernel
// inside 168 registers without spills). It adds in pairs: (a, a) + (b[j], b[j+1]) with one packed
// fp32 add (__fadd2_rn, round-to-nearest like the scalar add), and merges four candidates per
// accumulator with two 3-input max steps.
// Warp programs: the lane table groups the tasks by kind, one program per warp (r0_tables.inc).
// Tasks with kb == bi (A block on the diagonal) skip the k pairs a row meets only below the
// subdiagonal, tasks with kb == bj (shifted B block on the diagonal) skip the column pairs a k pair
// meets only below the diagonal, tasks with both skip both; the skipped candidates are all -inf,
// so every maximum is unchanged, and those warps issue 92, 80 and 49 of the 128 steps of a full
// task. At the end of a job the partial maxima of all tasks first meet in a shared
// tile of the cell's blocks (shared atomicMax; blocks at a pitch of 65 words so the lanes of a
// warp hit distinct banks), then the tile merges into F(i1, j1) with coalesced global atomicMax,
// consecutive lanes on consecutive words (max on the int bit patterns is exact: all values are
// >= +0; -inf partials and +0 entries are skipped).
#pragma once
#include <cstdint>

#include "bpmax_kernels.cuh"

namespace bpmax {

// one job: cell (i1, i1+d) of pair `pair`, k1 offset pairs p in [p0, p1) (offsets w = p and d-1-p)
struct R0Job {
    int pair, i1, p0, p1;
};

__host__ __device__ __forceinline__ int r0_job_items(const R0Job &j, int d)
{
    const int P = (d + 1) / 2;
    return 2 * (j.p1 - j.p0) - (((d & 1) && j.p1 == P) ? 1 : 0);
}
__host__ __device__ __forceinline__ int r0_item_offset(const R0Job &j, int d, int n)
{
    const int p = j.p0 + (n >> 1);
    return (n & 1) ? d - 1 - p : p;
}

// Shape variant V of the kernel for width class NB (a tunable of the schedule; results identical):
//   V = 0  three CTAs per SM (four for the 96-thread NB = 7), 168 registers, a 2..4-stage ring;
//   V = 1  two CTAs per SM (three below 128 threads), up to 255 registers, a ring of up to 6 stages.
template <int NB, int V = 0>
struct R0Cfg {
    static constexpr int NP = 8 * NB;
    static constexpr int THREADS = R0_TAB_THREADS[NB];
    static constexpr int G = R0_TAB_ITEMS[NB];              // items per iteration
    static constexpr int IMG = R0_TAB_COLBASE[NB][NB];      // chunks per cell image
    static constexpr int ITEM = 2 * IMG + R0_TAB_IPAD[NB];  // A image, B image, pad (chunks)
    static constexpr int STAGE = G * ITEM;                  // chunks
    static constexpr int STAGE_BYTES = STAGE * 16;
    static constexpr int NBLK = NB * (NB + 1) / 2;
    static constexpr int RED_WORDS = 65 * NBLK;             // job-merge tile, one 8x8 block per 65 words
    // shared-memory budget of the stages: 3 CTAs per SM; 4 for the 96-thread NB = 7 CTAs (their
    // registers allow it, and 12 resident warps beat a fourth stage)
    static constexpr int STAGE_BUDGET =
        (V == 1 ? (THREADS <= 96 ? 74 : 112) : (NB == 7 ? 55 : 75)) * 1024 - 4 * RED_WORDS - 4 * NBLK - 64;
    static constexpr int MAX_STAGES = V == 1 ? 6 : 4;
    static constexpr int STAGES = STAGE_BYTES * MAX_STAGES <= STAGE_BUDGET
                                      ? MAX_STAGES
                                      : (STAGE_BYTES * 4 <= STAGE_BUDGET ? 4 : (STAGE_BYTES * 3 <= STAGE_BUDGET ? 3 : 2));
    static constexpr int ITEM_TX = 2 * IMG * 16;            // bytes landing per item
    static constexpr int MINB = V == 1 ? (THREADS <= 64 ? 4 : (THREADS <= 96 ? 3 : 2))
                                       : (THREADS <= 64 ? 6 : (THREADS <= 96 ? 4 : 3));
    // shared memory: stages, merge tile, block offsets, one mbarrier per stage (byte offsets)
    static constexpr int OFF_RED = STAGES * STAGE_BYTES;
    static constexpr int OFF_DST = OFF_RED + 4 * RED_WORDS;
    static constexpr int OFF_BAR = (OFF_DST + 4 * NBLK + 15) / 16 * 16;
    static constexpr int OFF_CNT = OFF_BAR + 8 * STAGES;  // per stage: warps done with it
    static constexpr int OFF_ARM = OFF_CNT + 4 * STAGES;  // per stage: phases armed (expect_tx) so far
    static constexpr size_t SMEM = (size_t)OFF_ARM + 4 * STAGES;
    static constexpr int WARPS = THREADS / 32;
    // warp program of each warp, 2 bits per warp (0 full task, 1 diagonal A, 2 diagonal B, 3 both)
    static constexpr unsigned ROLE_BITS = R0_TAB_ROLE[NB][0] | R0_TAB_ROLE[NB][1] << 2 | R0_TAB_ROLE[NB][2] << 4 |
                                          R0_TAB_ROLE[NB][3] << 6 | R0_TAB_ROLE[NB][4] << 8 | R0_TAB_ROLE[NB][5] << 10 |
                                          R0_TAB_ROLE[NB][6] << 12 | R0_TAB_ROLE[NB][7] << 14;
    static_assert(STAGE_BYTES % 16 == 0 && OFF_RED % 16 == 0 && OFF_BAR % 8 == 0, "shared-memory alignment");
    static_assert(SMEM <= 227 * 1024, "shared memory per CTA");
};

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(unsigned bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// Control of the bounded waits of the product kernels (kernel argument, one per launch).
//   err:      device word set to 1 when a wait gives up (read by the host: BPMAX_ETIMEOUT)
//   wait_ns:  how long one wait may poll, in %globaltimer nanoseconds
//   inject:   1 = issue no operand copies at all, so the first wait of every CTA runs out with no
//             copy in flight (the host's test of the timeout path); 0 in every ordinary fill
struct WaitCtl {
    int *err;
    unsigned long long wait_ns;
    int inject;
};

__device__ __forceinline__ unsigned long long globaltimer_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ bool mbar_try(unsigned bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait for the completion of phase `parity` of an mbarrier: up to 1024 polls, then polls
// until the phase completes or limit_ns have passed; false when the limit ran out. (The plain
// polls keep the timer reads out of the common case, where the phase completes within them.)
__device__ __noinline__ bool mbar_wait_slow(unsigned bar, unsigned parity, unsigned long long limit_ns)
{
    const unsigned long long t0 = globaltimer_ns();
    while (!mbar_try(bar, parity))
        if (globaltimer_ns() - t0 > limit_ns) return false;
    return true;
}
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity, unsigned long long limit_ns)
{
    for (int tries = 0; tries < 1024; ++tries)
        if (mbar_try(bar, parity)) return true;
    return mbar_wait_slow(bar, parity, limit_ns);
}
// after a timeout: waits, bounded, for the last armed phase of every stage (one thread)
__device__ __noinline__ void mbar_drain(const uint64_t *bars, const int *armed, int stages, unsigned long long limit_ns)
{
    for (int s = 0; s < stages; ++s)
        if (armed[s] > 0) mbar_wait_slow(smem_u32(bars + s), (unsigned)(armed[s] - 1) & 1u, limit_ns);
}
// global -> shared bulk copy on the TMA engine (16-byte aligned addresses, size a multiple of 16)
__device__ __forceinline__ void bulk_g2s(unsigned dst, const void *src, unsigned bytes, unsigned bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

// One lane's task over one item: acc[i][j] = max over the task's k of A[i][k] + Bs[k][j].
// ROLE 0 (full) evaluates all 8 k; ROLE 1 (A block on the diagonal, kb == bi) evaluates the k
// pair p = (2p, 2p+1) only for rows i <= 2p+2, since A[i][k] = -inf for k < i-1; ROLE 2 (shifted B
// block on the diagonal, kb == bj) evaluates k pair p only for column pairs jp >= p, since
// Bs[k][j] = -inf for k > j; ROLE 3 (both blocks on the diagonal) applies both limits. The
// skipped candidates are all -inf, so the maxima are unchanged.
template <int ROLE>
__device__ __forceinline__ bool r0_pair_used(int i, int jp, int p)
{
    return ((ROLE & 1) == 0 || i <= 2 * p + 2) && ((ROLE & 2) == 0 || jp >= p);
}
template <int ROLE>
__device__ __forceinline__ void r0_task(const float *__restrict__ As, const float *__restrict__ Bs, float (&acc)[8][8])
{
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        float2 bv[4][4];  // bv[k][jp] = (Bs[4q+k][2jp], Bs[4q+k][2jp+1])
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int row = 4 * q + k, ro = 8 * row + (row == 7 ? 4 : 0);  // row 7: next block / S1 piece
            if (r0_pair_used<ROLE>(0, 0, 2 * q + k / 2) || r0_pair_used<ROLE>(0, 1, 2 * q + k / 2)) {  // row 0 widest
                const float4 t0 = *reinterpret_cast<const float4 *>(Bs + ro);
                bv[k][0] = make_float2(t0.x, t0.y); bv[k][1] = make_float2(t0.z, t0.w);
            }
            const float4 t1 = *reinterpret_cast<const float4 *>(Bs + ro + 4);
            bv[k][2] = make_float2(t1.x, t1.y); bv[k][3] = make_float2(t1.z, t1.w);
        }
        // one A row at a time: the row's 4 operands are live only for its 32 candidates
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            if (!r0_pair_used<ROLE>(i, 3, 2 * q) && !r0_pair_used<ROLE>(i, 3, 2 * q + 1)) continue;
            const float4 t = *reinterpret_cast<const float4 *>(As + 8 * i + 4 * q);
            const float av[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
            for (int jp = 0; jp < 4; ++jp) {
                const bool u0 = r0_pair_used<ROLE>(i, jp, 2 * q), u1 = r0_pair_used<ROLE>(i, jp, 2 * q + 1);
                if (u0 && u1) {
                    const float2 s0 = __fadd2_rn(make_float2(av[0], av[0]), bv[0][jp]);
                    const float2 s1 = __fadd2_rn(make_float2(av[1], av[1]), bv[1][jp]);
                    const float2 s2 = __fadd2_rn(make_float2(av[2], av[2]), bv[2][jp]);
                    const float2 s3 = __fadd2_rn(make_float2(av[3], av[3]), bv[3][jp]);
                    acc[i][2 * jp] = fmax3(fmax3(acc[i][2 * jp], s0.x, s1.x), s2.x, s3.x);
                    acc[i][2 * jp + 1] = fmax3(fmax3(acc[i][2 * jp + 1], s0.y, s1.y), s2.y, s3.y);
                } else if (u0 || u1) {
                    const int k0 = u0 ? 0 : 2;
                    const float2 s0 = __fadd2_rn(make_float2(av[k0], av[k0]), bv[k0][jp]);
                    const float2 s1 = __fadd2_rn(make_float2(av[k0 + 1], av[k0 + 1]), bv[k0 + 1][jp]);
                    acc[i][2 * jp] = fmax3(acc[i][2 * jp], s0.x, s1.x);
                    acc[i][2 * jp + 1] = fmax3(acc[i][2 * jp + 1], s0.y, s1.y);
                }
            }
        }
    }
}

template <int NB, int V = 0>
__global__ void __launch_bounds__(R0Cfg<NB, V>::THREADS, R0Cfg<NB, V>::MINB)
r0_kernel(const R0Job *__restrict__ jobs, int njobs, const PairDesc *__restrict__ pairs, float *__restrict__ F, int d,
          WaitCtl ctl)
{
    using C = R0Cfg<NB, V>;
    constexpr int S = C::STAGES;
    constexpr long long CELL = 4LL * C::IMG;
    extern __shared__ __align__(128) float r0sm[];
    float *smem = r0sm;
    int *red = reinterpret_cast<int *>(reinterpret_cast<char *>(smem) + C::OFF_RED);      // job-merge tile
    int *red_dst = reinterpret_cast<int *>(reinterpret_cast<char *>(smem) + C::OFF_DST);  // float offset of each
                                                                                          // block in a cell image
    uint64_t *bars = reinterpret_cast<uint64_t *>(reinterpret_cast<char *>(smem) + C::OFF_BAR);
    int *done_cnt = reinterpret_cast<int *>(reinterpret_cast<char *>(smem) + C::OFF_CNT);
    int *armed = reinterpret_cast<int *>(reinterpret_cast<char *>(smem) + C::OFF_ARM);  // phases armed per stage
    const int tid = threadIdx.x;
    int jid = blockIdx.x;
    if (jid >= njobs) return;

    if (tid == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(smem_u32(bars + s), 1);
            done_cnt[s] = 0;
            armed[s] = 0;
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int q = tid; q < C::RED_WORDS; q += C::THREADS) red[q] = 0;  // +0: below every partial maximum
    if (tid < C::NBLK) {
        int bi_ = 0, bj_ = tid;
        while (bj_ >= NB - bi_) { bj_ -= NB - bi_; ++bi_; }
        bj_ += bi_;
        red_dst[tid] = 4 * (c_img_colbase[NB][bj_] + 17 * bi_);
    }

    // the warp's program (uniform over its lanes) and this thread's task
    const int role = (int)(C::ROLE_BITS >> (2 * (tid >> 5))) & 3;
    const unsigned char *lt = c_r0_lane[NB - 1][tid];
    const bool has_task = lt[0] != 255;
    const int tg = has_task ? lt[0] : 0, bi = lt[1], bj = lt[2], kb = lt[3];
    int a_off = 0, b_off = 0, r3_off = 0, red_off = 0;
    if (has_task) {
        red_off = 65 * (bi * NB - bi * (bi - 1) / 2 + (bj - bi));       // block (bi, bj) of the merge tile
        a_off = 4 * (c_img_colbase[NB][kb] + 17 * bi);                 // A block (bi, kb), row 0
        b_off = 4 * (C::IMG + c_img_colbase[NB][bj] + 17 * kb + 2);     // shifted B block (kb, bj), row 0
        r3_off = 4 * (C::IMG + c_img_colbase[NB][bj] + 17 * bi);        // B row 8bi, columns 8bj..
    }
    constexpr int s1_off = 8;  // A[1][0] = S1(i1,k1): column 0, block 0, row 1
    __syncthreads();  // mbarrier init visible

    const unsigned smem_base = smem_u32(smem);
    const int lane = tid & 31;
    // announces the bytes of iteration `it` of a job of `items` items on stage s's mbarrier (one
    // thread, before any copy of that iteration is issued), and counts the stage's armed phases
    auto expect = [&](int s, int items, int it) {
        const int valid = min(C::G, items - it * C::G);
        mbar_arrive_tx(smem_u32(bars + s), (unsigned)(valid * C::ITEM_TX));
        armed[s] += 1;
    };
    // The producer's current job and its pair's M and F_off, one copy per warp in shared memory,
    // refreshed when the warp's producer position moves to another job: a refill then issues its
    // copies without the two dependent global loads (job record, then pair descriptor) it would
    // otherwise wait for on every item (positions stay indices, not records in registers, which
    // the product tile needs). 1024x64: 778 -> 766 ms per fill.
    __shared__ R0Job pjob_sh[C::WARPS];
    __shared__ long long pfoff_sh[C::WARPS];
    __shared__ int pm_sh[C::WARPS];
    const int warp_id = tid >> 5;
    auto load_pjob = [&](int j_) {
        __syncwarp();  // every lane of the warp is done with the previous copy
        if (lane == 0) {
            const R0Job jb = jobs[j_];
            pjob_sh[warp_id] = jb;
            pm_sh[warp_id] = pairs[jb.pair].M;
            pfoff_sh[warp_id] = pairs[jb.pair].F_off;
        }
        __syncwarp();
    };
    // issues the copies (whole cell images) of iteration `it` of the producer's job (j, the warp's
    // copy) into stage s, spread over the threads me, me+count, ...
    auto issue = [&](int s, int j, int it, int me, int count) {
        const R0Job jb = pjob_sh[warp_id];
        const int M = pm_sh[warp_id], j1 = jb.i1 + d;
        const int valid = min(C::G, r0_job_items(jb, d) - it * C::G);
        const unsigned bar = smem_u32(bars + s);
        const float *Fp = F + pfoff_sh[warp_id];
        for (int o = me; o < 2 * valid; o += count) {
            const int g = o >> 1, k1 = jb.i1 + r0_item_offset(jb, d, it * C::G + g);
            const long long cell = (o & 1) ? cell_index(M, k1 + 1, j1) : cell_index(M, jb.i1, k1);
            bulk_g2s(smem_base + (unsigned)(s * C::STAGE_BYTES + (g * C::ITEM + (o & 1) * C::IMG) * 16), Fp + cell * CELL,
                     (unsigned)(C::IMG * 16), bar);
        }
    };

    // consumer position (job jid of `items` items, iteration it) and producer position (pj, pitems,
    // pit), S iterations ahead; every warp advances both the same way, so all agree on which
    // iteration each stage holds
    int items = r0_job_items(jobs[jid], d), it = 0;
    int pj = jid, pit = 0, pitems = items;
    auto advance = [&](int &j_, int &items_, int &it_) {
        if (++it_ * C::G >= items_) {
            it_ = 0;
            j_ += gridDim.x;
            if (j_ < njobs) items_ = r0_job_items(jobs[j_], d);
        }
    };
    // the producer's advance also refreshes the warp's copy of its job (warp-uniform)
    auto advance_p = [&]() {
        if (++pit * C::G >= pitems) {
            pit = 0;
            pj += gridDim.x;
            if (pj < njobs) {
                pitems = r0_job_items(jobs[pj], d);
                load_pjob(pj);
            }
        }
    };
    load_pjob(pj);
    if (tid == 0 && !ctl.inject) {  // expected bytes of the first S iterations (every stage starts free)
        int j_ = pj, it_ = pit, items_ = pitems;
        for (int s = 0; s < S && j_ < njobs; ++s) {
            expect(s, items_, it_);
            advance(j_, items_, it_);
        }
    }
    __syncthreads();
#pragma unroll 1
    for (int s = 0; s < S; ++s)
        if (pj < njobs) {
            if (!ctl.inject) issue(s, pj, pit, tid, C::THREADS);
            advance_p();
        }

    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = NEG_INF;

    unsigned phase = 0;  // bit s: parity of stage s's next completion
    int stage = 0;
    // bad: a wait of this thread ran out. It then skips waits and work, arms and issues no more
    // copies, and the CTA leaves at the next job end after waiting (bounded) for the copies it
    // already issued, so none is left in flight into the shared memory of a finished CTA. This path
    // is best-effort: if those copies do not land within the limit either, the CTA leaves anyway.
    bool bad = false;
#pragma unroll 1
    while (true) {
        const bool active = has_task && it * C::G + tg < items;
        if (!bad && !mbar_wait(smem_u32(bars + stage), (phase >> stage) & 1u, ctl.wait_ns)) {
            atomicExch(ctl.err, 1);
            bad = true;
        }
        phase ^= 1u << stage;
        if (active && !bad) {
            const float *item = smem + (size_t)stage * C::STAGE * 4 + tg * C::ITEM * 4;
            const float *As = item + a_off, *Bs = item + b_off;
            if (role == 0)
                r0_task<0>(As, Bs, acc);
            else if (role == 1)
                r0_task<1>(As, Bs, acc);
            else if (role == 2)
                r0_task<2>(As, Bs, acc);
            else
                r0_task<3>(As, Bs, acc);
            if (kb == bi) {  // k = 8bi-1 term of row 8bi: S1(i1,k1) + B[8bi][j2]
                const float s1a = item[s1_off];
                const float4 r0 = *reinterpret_cast<const float4 *>(item + r3_off);
                const float4 r1 = *reinterpret_cast<const float4 *>(item + r3_off + 4);
                const float rv[8] = {r0.x, r0.y, r0.z, r0.w, r1.x, r1.y, r1.z, r1.w};
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[0][j] = fmaxf(acc[0][j], s1a + rv[j]);
            }
        }
        // the last warp done with this stage refills it with the iteration S ahead (not after a
        // timeout: the other warps' waits on the unarmed phase then run out too)
        __syncwarp();
        int last = 0;
        if (lane == 0) last = atomicAdd(done_cnt + stage, 1) == C::WARPS - 1;
        last = __shfl_sync(0xffffffffu, last, 0);
        if (last && pj < njobs && !__any_sync(0xffffffffu, bad)) {  // (test mode: every warp is bad by now)
            if (lane == 0) {
                done_cnt[stage] = 0;
                expect(stage, pitems, pit);
            }
            __syncwarp();
            issue(stage, pj, pit, lane, 32);
        } else if (last && lane == 0) {
            done_cnt[stage] = 0;
        }
        if (pj < njobs) advance_p();
        if (++it * C::G >= items) {  // job done: merge the partial maxima of all tasks into F(i1, i1+d)
            const R0Job job = jobs[jid];
            const PairDesc pd = pairs[job.pair];
            if (has_task) {
#pragma unroll
                for (int i = 0; i < 8; ++i)
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const int i2 = 8 * bi + i, j2 = 8 * bj + j;
                        const int v = __float_as_int(acc[i][j]);
                        if (i2 <= j2 && j2 < pd.N && v > 0) atomicMax(red + red_off + 8 * i + j, v);
                        acc[i][j] = NEG_INF;
                    }
            }
            if (__syncthreads_or(bad)) {  // no thread arms or issues from here on
                if (tid == 0) mbar_drain(bars, armed, S, ctl.wait_ns);
                return;
            }
            int *out = reinterpret_cast<int *>(F + pd.F_off + cell_index(pd.M, job.i1, job.i1 + d) * CELL);
            for (int e = tid; e < 64 * C::NBLK; e += C::THREADS) {
                const int q = e >> 6, w = e & 63;
                const int v = red[65 * q + w];
                if (v > 0) {
                    atomicMax(out + red_dst[q] + w, v);
                    red[65 * q + w] = 0;
                }
            }
            __syncthreads();  // the tile is clear before any warp merges its next job into it
            jid += gridDim.x;
            if (jid >= njobs) break;
            items = r0_job_items(jobs[jid], d);
            it = 0;
        }
        stage = (stage + 1) % S;
    }
}

}  // namespace bpmax
