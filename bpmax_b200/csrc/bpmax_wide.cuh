// bpmax_wide.cuh -- the R0 + R3 + R4 product kernel for inner tables stored as tile images
// (64 < Np <= WIDE_TILE_MAX_NP, Np = 64 * NT; layout in bpmax_kernels.cuh).
//
// The triangular (max,+) product of one item of the width-64 kernel (bpmax_r0.cuh),
//   max_{k in [i2-1, j2]} A[i2][k] + Bs[k][j2]      (R0, and R3 / R4 through S1 on the subdiagonals)
// splits over tiles: output tile (BI, BJ) takes the k tiles KB in [BI, BJ], item (k1, KB) being
// A = tile (BI, KB) of F(i1, k1) and B = tile (KB, BJ) of F(k1+1, j1) (every k outside [i2-1, j2] meets
// a -inf below a diagonal, and the k = 64 BI - 1 term of tile row BI's first row is the R3 step of
// the width-64 kernel: S1(i1, k1) + B[64 BI][j2], B's local row 0). Items are of four kinds:
//   DD  BI = BJ (= KB): both diagonal tiles, exactly an item of the width-64 kernel (its lane table
//       and warp programs);
//   DA  KB = BI < BJ: A diagonal, B dense;   F  BI < KB < BJ: both dense;   DB  BI < KB = BJ: B diagonal.
// A job is one output tile of one outer cell and a range of k1 offset pairs (w, d-1-w) as in the
// width-64 kernel; for each k1 it walks KB = BI .. BJ. Per item two bulk copies (cp.async.bulk, the
// whole A tile image and the whole B tile image) land in a stage of a shared-memory ring counted on
// the stage's mbarrier, with the width-64 kernel's refill scheme (the last warp done with a stage
// refills it; no CTA barrier per item) and bounded waits. In off-diagonal jobs each lane owns one
// 8x8 micro-tile of the output tile (two lanes per micro-tile) and takes, per item, part of its k
// blocks (wide_tables.inc). At the end of a job every lane merges its partial maxima into the
// output tile with global atomicMax on the bit patterns (exact: every value is >= +0; -inf and +0
// partials are skipped), so jobs of one tile commute.
#pragma once
#include "bpmax_r0.cuh"

namespace bpmax {

// one job: output tile (BI, BJ) (tile = BI << 8 | BJ) of cell (i1, i1+d) of pair `pair`, k1 offset
// pairs p in [p0, p1) (offsets w = p and d-1-p, as R0Job)
struct R0JobW {
    int pair, i1, tile, p0, p1;
};

// Shape variants: STAGES = 2 keeps three CTAs per SM (168 registers), 3 two CTAs per SM.
template <int STAGES_>
struct WideCfg {
    static constexpr int THREADS = 128;
    static constexpr int STAGES = STAGES_;
    static constexpr int SLOT = WIDE_DENSE_CHUNKS;  // chunks of one operand slot (a dense image fits)
    static constexpr int STAGE_BYTES = 2 * SLOT * 16;
    static constexpr int OFF_BAR = STAGES * STAGE_BYTES;
    static constexpr int OFF_CNT = OFF_BAR + 8 * STAGES;
    static constexpr int OFF_ARM = OFF_CNT + 4 * STAGES;
    static constexpr size_t SMEM = (size_t)OFF_ARM + 4 * STAGES;
    static constexpr int MINB = STAGES <= 2 ? 3 : 2;  // CTAs per SM the shared memory allows
    static constexpr int WARPS = THREADS / 32;
    static_assert(STAGE_BYTES % 16 == 0 && OFF_BAR % 8 == 0, "shared-memory alignment");
    static_assert((SMEM + 1024) * MINB <= 228 * 1024, "shared memory per SM");
};

template <int STAGES>
__global__ void __launch_bounds__(128, WideCfg<STAGES>::MINB)
r0_wide_kernel(const R0JobW *__restrict__ jobs, int njobs, const PairDesc *__restrict__ pairs, float *__restrict__ F,
               int d, WaitCtl ctl)
{
    using C = WideCfg<STAGES>;
    constexpr int S = STAGES;
    extern __shared__ __align__(128) float wsm[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(reinterpret_cast<char *>(wsm) + C::OFF_BAR);
    int *done_cnt = reinterpret_cast<int *>(reinterpret_cast<char *>(wsm) + C::OFF_CNT);
    int *armed = reinterpret_cast<int *>(reinterpret_cast<char *>(wsm) + C::OFF_ARM);
    const int tid = threadIdx.x, lane = tid & 31;
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
    __syncthreads();

    const unsigned smem_base = smem_u32(wsm);
    auto job_items = [&](const R0JobW &jb) {
        return r0_job_items(R0Job{jb.pair, jb.i1, jb.p0, jb.p1}, d) * ((jb.tile & 0xff) - (jb.tile >> 8) + 1);
    };
    // the producer's current job and its pair's M, Np and F_off, one copy per warp in shared memory,
    // refreshed when the warp's producer position moves to another job (as in r0_kernel: no
    // dependent global loads per refill)
    __shared__ R0JobW pjob_sh[C::WARPS];
    __shared__ long long pfoff_sh[C::WARPS];
    __shared__ int pm_sh[C::WARPS], pnp_sh[C::WARPS];
    const int warp_id = tid >> 5;
    auto load_pjob = [&](int j_) {
        __syncwarp();  // every lane of the warp is done with the previous copy
        if (lane == 0) {
            const R0JobW jb = jobs[j_];
            pjob_sh[warp_id] = jb;
            pm_sh[warp_id] = pairs[jb.pair].M;
            pnp_sh[warp_id] = pairs[jb.pair].Np;
            pfoff_sh[warp_id] = pairs[jb.pair].F_off;
        }
        __syncwarp();
    };
    // arms stage s for item n of the producer's job (the warp's copy) and issues its two copies
    // (one thread)
    auto fill_stage = [&](int s, int n) {
        const R0JobW jb = pjob_sh[warp_id];
        const int M = pm_sh[warp_id];
        const int BI = jb.tile >> 8, BJ = jb.tile & 0xff, nkb = BJ - BI + 1, KB = BI + n % nkb, NT = pnp_sh[warp_id] >> 6;
        const int k1 = jb.i1 + r0_item_offset(R0Job{jb.pair, jb.i1, jb.p0, jb.p1}, d, n / nkb);
        const int j1 = jb.i1 + d;
        const long long CELL = wide_cell_floats(NT);
        const float *Fp = F + pfoff_sh[warp_id];
        const unsigned bar = smem_u32(bars + s);
        const int ab = 16 * (KB == BI ? WIDE_DIAG_CHUNKS : WIDE_DENSE_CHUNKS);
        const int bb = 16 * (KB == BJ ? WIDE_DIAG_CHUNKS : WIDE_DENSE_CHUNKS);
        mbar_arrive_tx(bar, (unsigned)(ab + bb));
        armed[s] += 1;
        const unsigned dst = smem_base + (unsigned)(s * C::STAGE_BYTES);
        bulk_g2s(dst, Fp + cell_index(M, jb.i1, k1) * CELL + wide_tile_off(NT, BI, KB), (unsigned)ab, bar);
        bulk_g2s(dst + 16 * C::SLOT, Fp + cell_index(M, k1 + 1, j1) * CELL + wide_tile_off(NT, KB, BJ), (unsigned)bb,
                 bar);
    };

    // consumer position (job jid, item it of items) and producer position S items ahead
    int items = job_items(jobs[jid]), it = 0;
    int pj = jid, pit = 0, pitems = items;
    // the producer's advance (every warp the same way) also refreshes the warp's copy of its job
    auto advance_p = [&]() {
        if (++pit >= pitems) {
            pit = 0;
            pj += gridDim.x;
            if (pj < njobs) {
                pitems = job_items(jobs[pj]);
                load_pjob(pj);
            }
        }
    };
    load_pjob(pj);
    for (int s = 0; s < S; ++s)
        if (pj < njobs) {
            if (tid == 0 && !ctl.inject) fill_stage(s, pit);
            advance_p();
        }

    // the lane's task: DD jobs use the width-64 kernel's lane table and warp programs (task (bi, bj,
    // kb) packed as bi | bj << 4 | kb << 8, or -1 for an idle lane); the other jobs the micro-tile
    // table of wide_tables.inc (bi | bj << 4 | h << 8)
    const int warp_role = (int)(R0Cfg<8>::ROLE_BITS >> (2 * (tid >> 5))) & 3;
    const int dd_task = c_r0_lane[7][tid][0] == 255
                            ? -1
                            : (c_r0_lane[7][tid][1] | c_r0_lane[7][tid][2] << 4 | c_r0_lane[7][tid][3] << 8);
    const int mt_task = c_tile_lane[tid][0] | c_tile_lane[tid][1] << 4 | c_tile_lane[tid][2] << 8;
    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = NEG_INF;

    unsigned phase = 0;
    int stage = 0;
    bool bad = false;  // as in r0_kernel: a wait ran out; no more copies, leave at the next job end
    int tile = jobs[jid].tile, kbi = 0;  // the job's output tile; k tile of the item = BI + kbi
#pragma unroll 1
    while (true) {
        const int BI = tile >> 8, BJ = tile & 0xff, KB = BI + kbi;
        if (!bad && !mbar_wait(smem_u32(bars + stage), (phase >> stage) & 1u, ctl.wait_ns)) {
            atomicExch(ctl.err, 1);
            bad = true;
        }
        phase ^= 1u << stage;
        if (!bad) {
            const float *As = wsm + (size_t)stage * (C::STAGE_BYTES / 4);
            const float *Bs = As + 4 * C::SLOT;
            if (BI == BJ) {  // DD: one task of the width-64 table per lane
                if (dd_task >= 0) {
                    const int bi = dd_task & 15, bj = (dd_task >> 4) & 15, kb = dd_task >> 8;
                    const float *a = As + 4 * (c_img_colbase[8][kb] + 17 * bi);
                    const float *b = Bs + 4 * (c_img_colbase[8][bj] + 17 * kb + 2);
                    if (warp_role == 0)
                        r0_task<0>(a, b, acc);
                    else if (warp_role == 1)
                        r0_task<1>(a, b, acc);
                    else if (warp_role == 2)
                        r0_task<2>(a, b, acc);
                    else
                        r0_task<3>(a, b, acc);
                    if (kb == bi) {  // k = 8bi-1 term of row 8bi: S1(i1,k1) + B[8bi][j2]
                        const float s1a = As[8];
                        const float *r3 = Bs + 4 * (c_img_colbase[8][bj] + 17 * bi);
                        const float4 r0 = *reinterpret_cast<const float4 *>(r3);
                        const float4 r1 = *reinterpret_cast<const float4 *>(r3 + 4);
                        const float rv[8] = {r0.x, r0.y, r0.z, r0.w, r1.x, r1.y, r1.z, r1.w};
#pragma unroll
                        for (int j = 0; j < 8; ++j) acc[0][j] = fmaxf(acc[0][j], s1a + rv[j]);
                    }
                }
            } else {
                const int bi = mt_task & 15, bj = (mt_task >> 4) & 15, h = mt_task >> 8;
                const bool a_diag = KB == BI, b_diag = KB == BJ;
                int k0 = 4 * h, n = 4;
                if (a_diag || b_diag) {
                    const int lo = a_diag ? bi : 0, cnt = a_diag ? 8 - bi : bj + 1, half = (cnt + 1) >> 1;
                    k0 = h == 0 ? lo : lo + half;
                    n = h == 0 ? half : cnt - half;
                }
                const float *bcol = Bs + 4 * ((b_diag ? c_img_colbase[8][bj] : c_wide_dense_colbase[bj]) + 2);
#pragma unroll 1
                for (int kb = k0; kb < k0 + n; ++kb)
                    r0_task<0>(As + 4 * ((a_diag ? c_img_colbase[8][kb] : c_wide_dense_colbase[kb]) + 17 * bi),
                               bcol + 4 * 17 * kb, acc);
                if (a_diag && h == 0) {  // kb == bi is the first block of this lane: the k = 8bi-1 term
                    const float s1a = As[8];
                    const float *r3 = bcol + 4 * (17 * bi - 2);
                    const float4 r0 = *reinterpret_cast<const float4 *>(r3);
                    const float4 r1 = *reinterpret_cast<const float4 *>(r3 + 4);
                    const float rv[8] = {r0.x, r0.y, r0.z, r0.w, r1.x, r1.y, r1.z, r1.w};
#pragma unroll
                    for (int j = 0; j < 8; ++j) acc[0][j] = fmaxf(acc[0][j], s1a + rv[j]);
                }
            }
        }
        // the last warp done with this stage refills it with the item S ahead (not after a timeout)
        __syncwarp();
        int last = 0;
        if (lane == 0) last = atomicAdd(done_cnt + stage, 1) == C::WARPS - 1;
        last = __shfl_sync(0xffffffffu, last, 0);
        if (last) {
            const bool refill = pj < njobs && !__any_sync(0xffffffffu, bad);  // (test mode: every warp is bad)
            if (lane == 0) {
                done_cnt[stage] = 0;
                if (refill) fill_stage(stage, pit);
            }
        }
        if (pj < njobs) advance_p();
        if (++kbi > BJ - BI) kbi = 0;
        if (++it >= items) {  // job done: merge the partial maxima into the output tile
            const R0JobW job = jobs[jid];
            const PairDesc pd = pairs[job.pair];
            const int NT = pd.Np >> 6;
            float *out = F + pd.F_off + cell_index(pd.M, job.i1, job.i1 + d) * wide_cell_floats(NT) +
                         wide_tile_off(NT, BI, BJ);
            const int task = BI == BJ ? dd_task : mt_task;
            if (task >= 0) {
                const int bi = task & 15, bj = (task >> 4) & 15;
                int *o = reinterpret_cast<int *>(out) +
                         4 * ((BI == BJ ? c_img_colbase[8][bj] : c_wide_dense_colbase[bj]) + 17 * bi);
#pragma unroll
                for (int i = 0; i < 8; ++i)
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const int i2 = 64 * BI + 8 * bi + i, j2 = 64 * BJ + 8 * bj + j;
                        const int v = __float_as_int(acc[i][j]);
                        if (i2 <= j2 && j2 < pd.N && v > 0) atomicMax(o + 8 * i + j, v);
                        acc[i][j] = NEG_INF;
                    }
            }
            if (__syncthreads_or(bad)) {  // no thread arms or issues from here on
                if (tid == 0) mbar_drain(bars, armed, S, ctl.wait_ns);
                return;
            }
            jid += gridDim.x;
            if (jid >= njobs) break;
            const R0JobW nx = jobs[jid];
            items = job_items(nx);
            tile = nx.tile;
            it = 0;
            kbi = 0;
        }
        stage = (stage + 1) % S;
    }
}

}  // namespace bpmax
