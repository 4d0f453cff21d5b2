// bpmax_engine.cu -- host side of the B200 BPMax fill: device arenas, the outer-diagonal
// schedule, CUDA-graph capture, and the C ABI declared in include/bpmax_gpu.h.
//
// Schedule of one fill (any number of pairs of uneven lengths, batched on one stream):
//   clear F; single-strand tables S1, S2 of every pair;
//   for d = 0 .. max(M)-1:                     (outer wavefront over j1-i1, V3/bpmax.c:300-323)
//     R0+R3+R4 product kernel over the cells (i1, i1+d) of every pair with M > d: jobs of k1
//       offset pairs (w, d-1-w), ordered by offset pair so both uses of a table meet in L2;
//     finalize kernel over the same cells (init, SW1, inner R1/R2/SW2 wavefront, FT copy).
// The whole sequence is captured once per shape as a CUDA graph and replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <set>
#include <string>
#include <vector>

#include "../../include/bpmax_gpu.h"
#include "bpmax_kernels.cuh"
#include "bpmax_kernels_large.cuh"
#include "bpmax_r0.cuh"
#include "bpmax_adjoint.cuh"
#include "bpmax_r0only.cuh"
#include "bpmax_wide.cuh"
#include "bpmax_persist.cuh"

using namespace bpmax;

namespace {

// schedule tunables in key order: pairs per job, merge cost, class streams, product shape variant,
// tile-product stages, class shares, persistent fill
using Tuned = std::array<int, 7>;

constexpr int MAX_SMALL_NP = 64;
constexpr int MAX_CLASS_STREAMS = 8;  // side streams for the per-width-class chains of a batch
constexpr int MAX_NP = 4096;

// inner table width of a strand-2 length: multiples of 8 up to 64, then multiples of 64
int padded_width(int N) { return N <= MAX_SMALL_NP ? std::max(8, (N + 7) / 8 * 8) : (N + 63) / 64 * 64; }

// Offset pairs per product job on a diagonal with `cells` cells of P2 offset pairs each, for
// `resident` CTAs that each take every resident-th job. The launch lasts about
// ceil(jobs / resident) job lengths, a job of q pairs being 2q items plus one merge
// (`merge_items` items' worth): pick the chunk count that minimises that.
long long r0_pairs_per_job(long long cells, long long P2, long long resident, long long qmin, long long qmax,
                           long long merge_items)
{
    long long best_q = std::max(qmin, std::min(qmax, P2)), best_cost = -1;
    for (long long nch = 1; nch <= std::min<long long>(P2, 64); ++nch) {
        const long long q = std::max(qmin, std::min(qmax, (P2 + nch - 1) / nch));
        const long long jobs = cells * ((P2 + q - 1) / q);
        const long long cost = (jobs + resident - 1) / resident * (2 * q + merge_items);
        if (best_cost < 0 || cost < best_cost) {
            best_cost = cost;
            best_q = q;
        }
    }
    return best_q;
}

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
};

struct Plan {
    std::vector<int> Ms, Ns;
    std::vector<PairDesc> pairs;
    long long F_floats = 0, S_floats = 0;
    bool any_large = false;  // some pair has Np > WIDE_TILE_MAX_NP (row-major tables + FT)
    int bases_bytes = 0;
    int maxM = 0;
    // per diagonal and Np class (index NB-1): ranges in the job arrays
    // np = inner table width class; part (product launches): 0 = reads only diagonals <= d-2,
    // 1 = reads diagonal d-1 too
    // cap: at most this many CTAs (0: as many as are resident), from the class shares
    struct Launch { int d, np, first, count, s1_first = 0, s1_count = 0, part = 1, cap = 0; };
    std::vector<Launch> r0_launches, fin_launches;
    std::vector<R0Job> r0_jobs;
    std::vector<R0JobL> r0l_jobs;  // jobs of launches with np > WIDE_TILE_MAX_NP (first/count index this array)
    std::vector<R0JobW> r0w_jobs;  // jobs of launches with tile-image tables (first/count index this array)
    std::vector<CellJob> cell_jobs;
    std::vector<int> classes;  // distinct inner widths, ascending
    int pairs_per_job = 0, merge_items = 0, class_streams = 1;  // tunables the plan was built with
    int r0_variant = 0, wide_stages = 2, class_share = 0, persist = 0;
    bool r0_only = false;  // R0-only double max-plus (bpmax_gpu_r0_only) instead of the BPMax fill
    bool split = true;     // the product's offset pair 0 may run as its own launch (one-class plans)
    std::vector<cudaEvent_t> diag_ev;  // one pair only: outer diagonal d finalized (recorded by the graph)
    // persistent fill (one launch per width class walking the diagonals with dependency counters):
    // the work queues of all classes back to back, each class's range and CTA count
    bool persistent = false, copyout = false;
    RefOut ref{nullptr, 0, 0};  // finalize launches also write the reference layout (bpmax_gpu_fill)
    std::vector<PItem> pitems;
    struct PClass { int np, first, count, ctas; };
    std::vector<PClass> pclasses;
    std::vector<int> prod_need;  // per cell (PairDesc::cell_base + cell): product jobs
    int n_counters = 0;          // per-diagonal counters of all pairs
    cudaGraphExec_t graph = nullptr;
    long launches = 0;
};

}  // namespace

struct bpmax_ctx {
    int device = 0;
    int sms = 148;
    cudaStream_t stream = nullptr;
    cudaStream_t class_stream[8] = {};  // MAX_CLASS_STREAMS
    cudaStream_t aux_stream = nullptr;  // reference-layout conversion and copy-out, overlapped with the fill
    cudaEvent_t fork_ev = nullptr, join_ev[8] = {};
    // per width-class chain: a side stream for the product part that reads only diagonals <= d-2,
    // its completion event, and the chain's finalize events of the last two diagonals
    cudaStream_t side_stream[8] = {};
    cudaEvent_t side_done_ev[8] = {}, fin_ev[8][2] = {}, side_join_ev[8] = {};
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    Weights W;
    std::string err;
    DevBuf F, FT, S, bases, pairs, r0jobs, r0ljobs, r0wjobs, celljobs, scores, conv, tbstack, grads, tbstatus, errflag;
    DevBuf r0vals;         // R0-only mode: seq1 then seq2 of the pair, as floats
    DevBuf pq, pcnt, pneed;  // persistent fill: work queue; counters (class heads, diagonals, cells); jobs per cell
    bool copyout = false;    // the next fill copies the reference layout out per diagonal (graph path)
    RefOut want_ref{nullptr, 0, 0};  // the next fill's finalize also writes the reference layout there
    DevBuf refdev;                   // that reference layout, diagonal-major
    bool r0_only = false;  // mode of the next prepare()
    // schedule of the next prepare(): with the reference-layout copy-out running beside the fill
    // (bpmax_gpu_fill), the unsplit product leaves the SMs the row conversions need
    bool allow_split = true;
    int r0_occ_v[2][9] = {};  // resident product CTAs per SM, per shape variant and width class NB
    int wide_occ[4] = {};     // resident tile-product CTAs per SM, per stage count
    // schedule tunables (bpmax_gpu_set_tuning / bpmax_gpu_autotune); a plan is built with the
    // values current at build time, or with the values an autotune run stored for its shapes
    int r0_pairs_per_job = 1 << 20;                 // upper bound of k1 offset pairs per product job
    int r0_merge_items = 2;                         // cost of one job merge, in items, for job sizing
    int class_streams = 1;                          // run the width classes of a batch on parallel streams
    int r0_variant = 0;                             // shape variant of the width-64 product kernel (0 or 1)
    int wide_stages = 2;                            // shared-memory stages of the tile-image product (2 or 3)
    int class_share = 0;                            // cap each width class's product CTAs by its share of the work
    int persist = 0;  // width classes <= 64 by the persistent kernel: 0 no, 1 side by side, 2 one after another
    int persist_occ[9] = {};                        // resident persistent-fill CTAs per SM, per width class
    // bounded waits of the product kernels: time limit of one wait, and the one-shot test mode in
    // which the next fill's product kernels issue no copies (their first waits run out)
    unsigned long long wait_ns = 4000000000ULL;
    bool inject_wait_timeout = false;
    std::map<std::vector<int>, Tuned> tuned;  // shape signature (Ms then Ns) -> tunables
    float *host_stage[2] = {nullptr, nullptr};
    size_t host_stage_bytes = 0;
    cudaEvent_t stage_ev[2] = {nullptr, nullptr};
    Plan plan;
    bool plan_valid = false;
    float last_ms = 0.f;
    long last_launches = 0;
};

namespace {

int fail(bpmax_ctx *ctx, int status, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (ctx) ctx->err = buf;
    return status;
}

#define CK(call)                                                                                        \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess)                                                                          \
            return fail(ctx, e_ == cudaErrorMemoryAllocation ? BPMAX_ENOMEM : BPMAX_ECUDA, "%s: %s (%s:%d)", \
                        #call, cudaGetErrorString(e_), __FILE__, __LINE__);                              \
    } while (0)

int ensure(bpmax_ctx *ctx, DevBuf &b, size_t bytes)
{
    if (b.bytes >= bytes) return BPMAX_OK;
    if (b.p) CK(cudaFree(b.p));
    b.p = nullptr;
    b.bytes = 0;
    size_t want = std::max(bytes, (size_t)256);
    CK(cudaMalloc(&b.p, want));
    b.bytes = want;
    return BPMAX_OK;
}

WaitCtl wait_ctl(const bpmax_ctx *ctx)
{
    return WaitCtl{(int *)ctx->errflag.p, ctx->wait_ns, ctx->inject_wait_timeout ? 1 : 0};
}

int weights_ok(const float *w)
{
    for (int t = 0; t < 12; ++t)
        if (!std::isfinite(w[t]) || w[t] < 0.0f || std::signbit(w[t])) return 0;
    return 1;
}

long long align64(long long x) { return (x + 63) / 64 * 64; }

// Builds the device layout and the per-diagonal job lists for the given pair shapes.
std::vector<int> shape_key(const std::vector<int> &Ms, const std::vector<int> &Ns)
{
    std::vector<int> k(Ms);
    k.insert(k.end(), Ns.begin(), Ns.end());
    return k;
}

// Work queue of the persistent fill, per width class: for d = 1, 2, ... the finalize items of
// diagonal d-1, then the product jobs of diagonal d with offset pairs >= 1, then the jobs of d for
// offset pair 0 (the only ones reading diagonal d-1); the finalize items of the last diagonal close
// it. Every item depends only on items before it (bpmax_persist.cuh), and the finalize of d-1 runs
// beside the long product group of d. Jobs of one group are ordered by pair chunk, then cell, as in
// the graph path. CTA counts: one class takes every resident CTA. Several classes either run one
// after another, each with every resident CTA (mode 2), or side by side (mode 1), each with a number
// of SMs proportional to its estimated time, so that all of them are resident at once.
void build_queue(bpmax_ctx *ctx, Plan &P)
{
    const int n = (int)P.pairs.size();
    long long ncells = 0;
    for (const auto &pd : P.pairs) ncells += (long long)pd.M * (pd.M + 1) / 2;
    P.prod_need.assign(ncells, 0);
    P.pitems.clear();
    P.pclasses.clear();
    // estimated CTA-microseconds per class: product items (one C(Np)+2T(Np) block each) and
    // finalizes, at the per-CTA costs of each width measured with this kernel on a B200, per SM
    // (divided by the CTAs one SM holds)
    static const double ITEM_US[9] = {0, 0.19, 0.30, 0.42, 0.65, 0.93, 1.2, 2.1, 2.1};
    static const double FIN_US[9] = {0, 4.0, 6.0, 9.0, 14.0, 24.0, 36.0, 72.0, 80.0};
    auto C3 = [](double x) { return x * (x * x - 1) / 6; };
    auto T2 = [](double x) { return x * (x + 1) / 2; };
    std::map<int, double> sm_time;
    double sm_tot = 0;
    for (const auto &pd : P.pairs) {
        const int NB = pd.Np / 8;
        const double t = (C3(pd.M) * ITEM_US[NB] + T2(pd.M) * FIN_US[NB]) / std::max(1, ctx->persist_occ[NB]);
        sm_time[pd.Np] += t;
        sm_tot += t;
    }
    std::map<int, int> sms_of;
    const bool side = P.classes.size() > 1 && P.persist == 1;
    if (side) {  // SMs per class, all classes resident at once (a margin of 2 SMs for uneven packing)
        const int budget = std::max((int)P.classes.size(), ctx->sms - 2);
        int used = 0;
        for (int np : P.classes) {
            sms_of[np] = std::max(1, (int)std::lround(budget * sm_time[np] / sm_tot));
            used += sms_of[np];
        }
        while (used > budget) {  // take the excess from the largest shares
            int big = P.classes[0];
            for (int np : P.classes)
                if (sms_of[np] > sms_of[big]) big = np;
            if (sms_of[big] <= 1) break;
            --sms_of[big];
            --used;
        }
    }
    for (int np : P.classes) {
        const int NB = np / 8, G = R0_TAB_ITEMS[NB];
        const int occ = std::max(1, ctx->persist_occ[NB]);
        const int ctas = side ? sms_of[np] * occ : occ * ctx->sms;
        const int first = (int)P.pitems.size();
        int maxM = 0;
        for (const auto &pd : P.pairs)
            if (pd.Np == np) maxM = std::max(maxM, pd.M);
        auto fin_items = [&](int e) {
            for (int p = 0; p < n; ++p)
                if (P.pairs[p].Np == np && P.pairs[p].M > e)
                    for (int i1 = 0; i1 < P.pairs[p].M - e; ++i1) P.pitems.push_back(PItem{p, i1, e, 0, 0, 1});
        };
        const long long qmin = std::max(1, (G + 1) / 2);
        for (int d = 1; d <= maxM; ++d) {
            const long long P2 = (d + 1) / 2;
            long long cells = 0;
            for (const auto &pd : P.pairs)
                if (pd.Np == np && pd.M > d) cells += pd.M - d;
            fin_items(d - 1);
            if (cells > 0 && P2 > 1) {  // offset pairs >= 1
                const long long q = r0_pairs_per_job(cells, P2 - 1, ctas, qmin, std::max<long long>(P.pairs_per_job, qmin),
                                                     P.merge_items);
                for (long long c0 = 1; c0 < P2; c0 += q)
                    for (int p = 0; p < n; ++p)
                        if (P.pairs[p].Np == np && P.pairs[p].M > d)
                            for (int i1 = 0; i1 < P.pairs[p].M - d; ++i1) {
                                P.pitems.push_back(PItem{p, i1, d, (int)c0, (int)std::min(c0 + q, P2), 0});
                                P.prod_need[P.pairs[p].cell_base + cell_index(P.pairs[p].M, i1, i1 + d)] += 1;
                            }
            }
            if (cells > 0)  // offset pair 0 (offsets 0 and d-1)
                for (int p = 0; p < n; ++p)
                    if (P.pairs[p].Np == np && P.pairs[p].M > d)
                        for (int i1 = 0; i1 < P.pairs[p].M - d; ++i1) {
                            P.pitems.push_back(PItem{p, i1, d, 0, 1, 0});
                            P.prod_need[P.pairs[p].cell_base + cell_index(P.pairs[p].M, i1, i1 + d)] += 1;
                        }
        }
        P.pclasses.push_back(Plan::PClass{np, first, (int)P.pitems.size() - first, ctas});
    }
}

int build_plan(bpmax_ctx *ctx, const std::vector<int> &Ms, const std::vector<int> &Ns, Plan &P)
{
    P = Plan();
    P.Ms = Ms;
    P.Ns = Ns;
    P.pairs_per_job = ctx->r0_pairs_per_job;
    P.merge_items = ctx->r0_merge_items;
    P.class_streams = ctx->class_streams;
    P.split = ctx->allow_split;
    P.r0_variant = ctx->r0_variant;
    P.wide_stages = ctx->wide_stages;
    P.class_share = ctx->class_share;
    P.persist = ctx->persist;
    const auto tu = ctx->tuned.find(shape_key(Ms, Ns));
    if (tu != ctx->tuned.end()) {
        P.pairs_per_job = tu->second[0];
        P.merge_items = tu->second[1];
        P.class_streams = tu->second[2];
        P.r0_variant = tu->second[3];
        P.wide_stages = tu->second[4];
        P.class_share = tu->second[5];
        P.persist = tu->second[6];
    }
    const int n = (int)Ms.size();
    long long f = 0, s = 0;
    int b = 0;
    for (int p = 0; p < n; ++p) {
        PairDesc pd{};
        pd.M = Ms[p];
        pd.N = Ns[p];
        pd.Np = padded_width(Ns[p]);
        if (pd.Np > MAX_NP) return fail(ctx, BPMAX_EINVAL, "strand-2 length %d > %d is not supported", Ns[p], MAX_NP);
        pd.F_off = f;
        f = align64(f + (long long)Ms[p] * (Ms[p] + 1) / 2 * cell_floats(pd.Np));
        if (pd.Np > WIDE_TILE_MAX_NP) P.any_large = true;
        pd.S1_off = s;
        s = align64(s + (long long)Ms[p] * Ms[p]);
        pd.S2_off = s;
        s = align64(s + (long long)pd.Np * pd.Np);
        pd.S2m_off = s;  // masked copies of S2 read by the inner wavefront
        s = align64(s + (long long)pd.Np * pd.Np);
        pd.S2t_off = s;
        s = align64(s + (long long)pd.Np * pd.Np);
        pd.S2d_off = s;
        if (pd.Np > MAX_SMALL_NP) s = align64(s + (long long)pd.Np * (pd.Np + 1) / 2);  // triangular S2D
        pd.seq1_off = b;
        b += Ms[p];
        pd.seq2_off = b;
        b += Ns[p];
        pd.cnt_off = P.n_counters;
        P.n_counters += Ms[p];
        pd.cell_base = p == 0 ? 0 : P.pairs.back().cell_base + (long long)P.pairs.back().M * (P.pairs.back().M + 1) / 2;
        P.pairs.push_back(pd);
        P.maxM = std::max(P.maxM, Ms[p]);
    }
    P.F_floats = f;
    P.S_floats = s;
    P.bases_bytes = b;
    std::vector<int> classes;
    for (const auto &pd : P.pairs) classes.push_back(pd.Np);
    std::sort(classes.begin(), classes.end());
    classes.erase(std::unique(classes.begin(), classes.end()), classes.end());
    P.classes = classes;
    // class shares: with several width classes on parallel graph branches, a product launch of one
    // class may hold every SM until its last job ends, so the branches run one after another. With
    // class shares on, each class's product launches take at most its share of the resident CTAs
    // (its share of the padded product terms, at least 1/16), so every branch keeps progressing.
    std::map<int, double> share;
    if (P.class_share && classes.size() > 1 && P.class_streams) {
        auto C3 = [](double x) { return x * (x * x - 1) / 6; };
        auto T2 = [](double x) { return x * (x + 1) / 2; };
        double tot = 0;
        for (const auto &pd : P.pairs) {
            const double w = C3(pd.M) * (C3(pd.Np) + 2 * T2(pd.Np));
            share[pd.Np] += w;
            tot += w;
        }
        for (auto &kv : share) kv.second = std::max(kv.second / tot, 1.0 / 16);
    }
    auto capped = [&](int np, long long resident) {
        const auto it = share.find(np);
        return it == share.end() ? resident : std::max(1LL, (long long)std::llround(resident * it->second));
    };
    // jobs, grouped by diagonal then inner width class
    const int target = 4 * ctx->sms;  // CTAs per diagonal launch worth splitting k1 for (wide tables)
    for (int d = 0; d < P.maxM; ++d) {
        for (int np : classes) {
            long long cells = 0;
            for (int p = 0; p < n; ++p)
                if (P.pairs[p].Np == np && Ms[p] > d) cells += Ms[p] - d;
            if (cells == 0) continue;
            Plan::Launch fl{d, np, (int)P.cell_jobs.size(), 0};
            for (int p = 0; p < n; ++p)
                if (P.pairs[p].Np == np && Ms[p] > d)
                    for (int i1 = 0; i1 < Ms[p] - d; ++i1) P.cell_jobs.push_back(CellJob{p, i1});
            fl.count = (int)P.cell_jobs.size() - fl.first;
            P.fin_launches.push_back(fl);
            if (d == 0) continue;
            if (np <= MAX_SMALL_NP) {
                // jobs of q offset pairs (w, d-1-w), ordered by pair chunk, then pair, then cell: the
                // two uses of a table (A of cell (a, a+d) at offset w, B of cell (a+w-d, a+w) at
                // offset d-1-w) fall in the same pair chunk
                const int NB = np / 8, G = R0_TAB_ITEMS[NB];
                const long long P2 = (d + 1) / 2;  // offset pairs per cell
                const long long resident =
                    capped(np, (long long)std::max(1, ctx->r0_occ_v[P.r0_variant][NB]) * ctx->sms);
                const long long qmin = std::max(1, (G + 1) / 2), qmax = std::max<long long>(P.pairs_per_job, qmin);
                // Offset pair 0 (offsets 0 and d-1) is the only one that reads diagonal d-1. In a plan
                // of one width class, where one iteration holds at most 2 items, it becomes its own
                // launch (part 1) and the other pairs (part 0, reading diagonals <= d-2) can run while
                // diagonal d-1 is finalized (several classes already overlap each other's finalize).
                const long long first_pair = (P.split && classes.size() == 1 && G <= 2 && P2 > 1) ? 1 : 0;
                if (first_pair) {
                    Plan::Launch rb{d, np, (int)P.r0_jobs.size(), 0};
                    rb.cap = share.empty() ? 0 : (int)resident;
                    for (int p = 0; p < n; ++p)
                        if (P.pairs[p].Np == np && Ms[p] > d)
                            for (int i1 = 0; i1 < Ms[p] - d; ++i1) P.r0_jobs.push_back(R0Job{p, i1, 0, 1});
                    rb.count = (int)P.r0_jobs.size() - rb.first;
                    P.r0_launches.push_back(rb);
                }
                const long long q = r0_pairs_per_job(cells, P2 - first_pair, resident, qmin, qmax, P.merge_items);
                Plan::Launch rl{d, np, (int)P.r0_jobs.size(), 0};
                rl.part = first_pair ? 0 : 1;
                rl.cap = share.empty() ? 0 : (int)resident;
                for (long long c0 = first_pair; c0 < P2; c0 += q)
                    for (int p = 0; p < n; ++p)
                        if (P.pairs[p].Np == np && Ms[p] > d)
                            for (int i1 = 0; i1 < Ms[p] - d; ++i1)
                                P.r0_jobs.push_back(R0Job{p, i1, (int)c0, (int)std::min(c0 + q, P2)});
                rl.count = (int)P.r0_jobs.size() - rl.first;
                P.r0_launches.push_back(rl);
                continue;
            }
            if (np <= WIDE_TILE_MAX_NP) {
                // tile images: one job per output tile (BI, BJ) of a cell and chunk of k1 offset pairs,
                // each tile's chunk sized so that jobs cost about the same: cost per offset pair in
                // warp task steps of both of its items, DD 3.3, DA and DB 12, F 16 per item
                const int NT = np / 64;
                const long long P2 = (d + 1) / 2;
                const long long resident = capped(np, (long long)std::max(1, ctx->wide_occ[P.wide_stages]) * ctx->sms);
                std::vector<std::pair<double, int>> tiles;  // (cost per offset pair, BI << 8 | BJ)
                double per_pair = 0;
                for (int BI = 0; BI < NT; ++BI)
                    for (int BJ = BI; BJ < NT; ++BJ) {
                        const double c = BI == BJ ? 2 * 3.3 : 2 * (24.0 + 16.0 * (BJ - BI - 1));
                        tiles.push_back({c, BI << 8 | BJ});
                        per_pair += c;
                    }
                std::stable_sort(tiles.begin(), tiles.end(), [](const auto &a, const auto &b) { return a.first > b.first; });
                const double total = (double)cells * P2 * per_pair;
                const double target = std::max(total / (3.0 * resident), 4.0 * 16.0);
                const size_t first = P.r0w_jobs.size();
                for (const auto &t : tiles) {
                    const long long q = std::max(1LL, std::min(P2, (long long)std::llround(target / t.first)));
                    for (long long c0 = 0; c0 < P2; c0 += q)
                        for (int p = 0; p < n; ++p)
                            if (P.pairs[p].Np == np && Ms[p] > d)
                                for (int i1 = 0; i1 < Ms[p] - d; ++i1)
                                    P.r0w_jobs.push_back(R0JobW{p, i1, t.second, (int)c0, (int)std::min(c0 + q, P2)});
                }
                // jobs of the same offset pairs together (both uses of a table meet in L2), heavy tiles first
                std::stable_sort(P.r0w_jobs.begin() + first, P.r0w_jobs.end(),
                                 [](const R0JobW &a, const R0JobW &b) { return a.p0 < b.p0; });
                Plan::Launch wl{d, np, (int)first, (int)(P.r0w_jobs.size() - first)};
                wl.cap = share.empty() ? 0 : (int)resident;
                P.r0_launches.push_back(wl);
                continue;
            }
            const int nbk = np / 64;
            const long long units = cells * (nbk * (nbk + 1) / 2);
            long long chunks = std::max(1LL, std::min((long long)d, (target + units - 1) / units));
            int csize = (int)((d + chunks - 1) / chunks);
            Plan::Launch rl{d, np, (int)P.r0l_jobs.size(), 0};
            for (int p = 0; p < n; ++p)
                if (P.pairs[p].Np == np && Ms[p] > d)
                    for (int i1 = 0; i1 < Ms[p] - d; ++i1)
                        for (int k = i1; k < i1 + d; k += csize) {
                            const int kb = std::min(k + csize, i1 + d);
                            // heavier blocks (more k' blocks) first
                            for (int D = nbk - 1; D >= 0; --D)
                                for (int BI = 0; BI + D < nbk; ++BI)
                                    P.r0l_jobs.push_back(R0JobL{p, i1, k, kb, (BI << 16) | (BI + D)});
                        }
            rl.count = (int)P.r0l_jobs.size() - rl.first;
            P.r0_launches.push_back(rl);
        }
    }
    // S1 of diagonal d+1 is computed by the finalize launch of diagonal d (same class)
    for (auto &fl : P.fin_launches)
        for (const auto &nx : P.fin_launches)
            if (nx.d == fl.d + 1 && nx.np == fl.np) { fl.s1_first = nx.first; fl.s1_count = nx.count; }
    // the persistent fill: width classes <= 64 only, not the R0-only mode, not the reference-layout
    // fill with its per-diagonal copy-out (both keep the graph of per-diagonal launches)
    P.copyout = ctx->copyout;
    P.persistent = P.persist && !ctx->r0_only && !ctx->copyout && P.classes.back() <= MAX_SMALL_NP;
    if (P.persistent) build_queue(ctx, P);
    return BPMAX_OK;
}

void launch_r0_large(bpmax_ctx *ctx, const Plan::Launch &L, cudaStream_t s)
{
    const int grid = std::min(L.count, 3 * ctx->sms);
    r0_large_kernel<<<grid, 128, WideShape::SMEM, s>>>(
        (const R0JobL *)ctx->r0ljobs.p + L.first, L.count, (const PairDesc *)ctx->pairs.p, (float *)ctx->F.p,
        (const float *)ctx->FT.p, (const float *)ctx->S.p, L.d);
}

template <int STAGES>
void launch_r0_wide_t(bpmax_ctx *ctx, const Plan::Launch &L, cudaStream_t s)
{
    const int grid = std::min(L.count, L.cap > 0 ? L.cap : std::max(1, ctx->wide_occ[STAGES]) * ctx->sms);
    r0_wide_kernel<STAGES><<<grid, WideCfg<STAGES>::THREADS, WideCfg<STAGES>::SMEM, s>>>(
        (const R0JobW *)ctx->r0wjobs.p + L.first, L.count, (const PairDesc *)ctx->pairs.p, (float *)ctx->F.p, L.d,
        wait_ctl(ctx));
}

void launch_r0_wide(bpmax_ctx *ctx, const Plan &P, const Plan::Launch &L, cudaStream_t s)
{
    if (P.wide_stages == 3)
        launch_r0_wide_t<3>(ctx, L, s);
    else
        launch_r0_wide_t<2>(ctx, L, s);
}

// the finalize of one launch of cells wider than 64; returns the number of kernel launches
int launch_fin_large(bpmax_ctx *ctx, const Plan::Launch &L, cudaStream_t s)
{
    const CellJob *jobs = (const CellJob *)ctx->celljobs.p + L.first;
    const CellJob *s1jobs = (const CellJob *)ctx->celljobs.p + L.s1_first;
    const PairDesc *pairs = (const PairDesc *)ctx->pairs.p;
    const uint8_t *bases = (const uint8_t *)ctx->bases.p;
    float *F = (float *)ctx->F.p, *S = (float *)ctx->S.p;
    if (L.np <= FIN_WIDE_MAX_NP) {
        constexpr int WW = FIN_WIDE_THREADS / 32;
        finalize_wide_kernel<<<L.count + (L.s1_count + WW - 1) / WW, FIN_WIDE_THREADS, fin_wide_smem(L.np), s>>>(
            jobs, L.count, s1jobs, L.s1_count, pairs, F, S, bases, ctx->W, L.d);
        return 1;
    }
    // row-major tables: start values, then per tile diagonal t the products over finished tiles and
    // the tiles' own wavefronts, then the SW1 pushes, the S1 slots and S1 of diagonal d+1
    float *FT = (float *)ctx->FT.p;
    const int nt32 = L.np / 32, NT = L.np / LT;
    int n = 0;
    if (L.count > 0) {
        large_init_kernel<<<dim3(nt32 * nt32, L.count), dim3(32, 8), 0, s>>>(jobs, pairs, F, FT, S, bases, ctx->W, L.d);
        ++n;
        for (int t = 0; t < NT; ++t) {
            if (t > 0) {
                large_tile_product_kernel<<<dim3(NT - t, L.count), 256, 0, s>>>(jobs, pairs, F, FT, S, L.d, t);
                ++n;
            }
            large_tile_local_kernel<<<dim3(NT - t, L.count), 256, LARGE_LOCAL_SMEM, s>>>(jobs, pairs, F, FT, S, bases,
                                                                                         ctx->W, L.d, t);
            ++n;
        }
    }
    const long long tile = (long long)L.np * L.np;
    const int chunks = (int)((tile + LARGE_FINAL_CHUNK - 1) / LARGE_FINAL_CHUNK);
    large_final_kernel<<<L.count * chunks + (L.s1_count + 7) / 8, 256, 0, s>>>(jobs, L.count, chunks, s1jobs, L.s1_count,
                                                                             pairs, F, FT, S, bases, ctx->W, L.d);
    return n + 1;
}

template <int NB, int V>
void launch_r0_v(bpmax_ctx *ctx, const Plan::Launch &L, cudaStream_t s)
{
    using C = R0Cfg<NB, V>;
    // resident CTAs (or the class's share of them); each loops over jobs
    const int grid = std::min(L.count, L.cap > 0 ? L.cap : std::max(1, ctx->r0_occ_v[V][NB]) * ctx->sms);
    r0_kernel<NB, V><<<grid, C::THREADS, C::SMEM, s>>>((const R0Job *)ctx->r0jobs.p + L.first, L.count,
                                                       (const PairDesc *)ctx->pairs.p, (float *)ctx->F.p, L.d,
                                                       wait_ctl(ctx));
}

template <int NB>
void launch_persist(bpmax_ctx *ctx, const PersistCtl &pc, int ctas, cudaStream_t s)
{
    fill_persistent_kernel<NB><<<ctas, R0Cfg<NB>::THREADS, R0Cfg<NB>::SMEM, s>>>(
        pc, (const PairDesc *)ctx->pairs.p, (float *)ctx->F.p, (float *)ctx->S.p, (const uint8_t *)ctx->bases.p, ctx->W,
        wait_ctl(ctx));
}

template <int NB>
void launch_r0(bpmax_ctx *ctx, const Plan &P, const Plan::Launch &L, cudaStream_t s)
{
    if (P.r0_variant == 1)
        launch_r0_v<NB, 1>(ctx, L, s);
    else
        launch_r0_v<NB, 0>(ctx, L, s);
}

template <int NB, int T>
void launch_fin_t(bpmax_ctx *ctx, const Plan::Launch &L, cudaStream_t s)
{
    using Sh = FinShape<8 * NB, T>;
    finalize_small_kernel<8 * NB, T><<<L.count + (L.s1_count + Sh::WARPS - 1) / Sh::WARPS, Sh::THREADS, Sh::SMEM, s>>>(
        (const CellJob *)ctx->celljobs.p + L.first, L.count, (const CellJob *)ctx->celljobs.p + L.s1_first, L.s1_count,
        (const PairDesc *)ctx->pairs.p, (float *)ctx->F.p, (float *)ctx->S.p, (const uint8_t *)ctx->bases.p, ctx->W,
        L.d, ctx->plan.ref);
}

template <int NB>
void launch_fin(bpmax_ctx *ctx, const Plan::Launch &L, cudaStream_t s)
{
    if constexpr (8 * NB >= 48) {
        if (L.count >= FIN_BULK_CELLS) return launch_fin_t<NB, FIN_BULK_THREADS>(ctx, L, s);
    }
    launch_fin_t<NB, fin_threads(8 * NB)>(ctx, L, s);
}

void launch_r0only_fin(bpmax_ctx *ctx, const Plan::Launch &L, cudaStream_t s)
{
    const CellJob *jobs = (const CellJob *)ctx->celljobs.p + L.first;
    const PairDesc *pd = (const PairDesc *)ctx->pairs.p;
    const float *vals = (const float *)ctx->r0vals.p;
    switch (L.np > MAX_SMALL_NP ? 0 : L.np / 8) {
    case 0:
        if (L.np <= WIDE_TILE_MAX_NP)
            r0only_finalize_tile_kernel<<<L.count, 256, 0, s>>>(jobs, pd, (float *)ctx->F.p, vals, L.d);
        else
            r0only_finalize_wide_kernel<<<dim3(L.count, L.np / R0ONLY_TILE), 256, 0, s>>>(jobs, pd, (float *)ctx->F.p,
                                                                                         (float *)ctx->FT.p, vals, L.d);
        break;
    case 1: r0only_finalize_small_kernel<8><<<L.count, 128, 0, s>>>(jobs, pd, (float *)ctx->F.p, vals, L.d); break;
    case 2: r0only_finalize_small_kernel<16><<<L.count, 128, 0, s>>>(jobs, pd, (float *)ctx->F.p, vals, L.d); break;
    case 3: r0only_finalize_small_kernel<24><<<L.count, 128, 0, s>>>(jobs, pd, (float *)ctx->F.p, vals, L.d); break;
    case 4: r0only_finalize_small_kernel<32><<<L.count, 128, 0, s>>>(jobs, pd, (float *)ctx->F.p, vals, L.d); break;
    case 5: r0only_finalize_small_kernel<40><<<L.count, 128, 0, s>>>(jobs, pd, (float *)ctx->F.p, vals, L.d); break;
    case 6: r0only_finalize_small_kernel<48><<<L.count, 128, 0, s>>>(jobs, pd, (float *)ctx->F.p, vals, L.d); break;
    case 7: r0only_finalize_small_kernel<56><<<L.count, 128, 0, s>>>(jobs, pd, (float *)ctx->F.p, vals, L.d); break;
    default: r0only_finalize_small_kernel<64><<<L.count, 128, 0, s>>>(jobs, pd, (float *)ctx->F.p, vals, L.d); break;
    }
}

// The product kernels, the small finalize and the persistent fill prefer the largest shared-memory
// carveout: an SM runs CTAs of different kernels side by side only when they use the same L1 /
// shared-memory split (parallel graph branches of a batch, the persistent launches of its width
// classes, the split product launches of one class).
template <typename K>
int prefer_smem(bpmax_ctx *ctx, K kernel)
{
    CK(cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    return BPMAX_OK;
}

template <int NB>
int set_smem_attr(bpmax_ctx *ctx)
{
    int st;
    if ((st = prefer_smem(ctx, r0_kernel<NB>)) || (st = prefer_smem(ctx, r0_kernel<NB, 1>)) ||
        (st = prefer_smem(ctx, finalize_small_kernel<8 * NB>)) || (st = prefer_smem(ctx, r0only_finalize_small_kernel<8 * NB>)))
        return st;
    if constexpr (8 * NB >= 48)
        if ((st = prefer_smem(ctx, finalize_small_kernel<8 * NB, FIN_BULK_THREADS>))) return st;
    if (NB == 8)
        if ((st = prefer_smem(ctx, r0_wide_kernel<2>)) || (st = prefer_smem(ctx, r0_wide_kernel<3>)) ||
            (st = prefer_smem(ctx, r0_large_kernel)))
            return st;
    // (the wide finalize kernels keep the driver's choice: their S2 reads live on the L1 that a
    // larger shared-memory carveout would take away, 389 vs 324 ms at 256x256)
    CK(cudaFuncSetAttribute(r0_kernel<NB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)R0Cfg<NB>::SMEM));
    CK(cudaFuncSetAttribute(r0_kernel<NB, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)R0Cfg<NB, 1>::SMEM));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ctx->r0_occ_v[1][NB], r0_kernel<NB, 1>, R0Cfg<NB, 1>::THREADS,
                                                     R0Cfg<NB, 1>::SMEM));
    CK(cudaFuncSetAttribute(finalize_small_kernel<8 * NB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)FinShape<8 * NB>::SMEM));
    if constexpr (8 * NB >= 48)
        CK(cudaFuncSetAttribute(finalize_small_kernel<8 * NB, FIN_BULK_THREADS>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)FinShape<8 * NB, FIN_BULK_THREADS>::SMEM));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ctx->r0_occ_v[0][NB], r0_kernel<NB>, R0Cfg<NB>::THREADS,
                                                     R0Cfg<NB>::SMEM));
    CK(cudaFuncSetAttribute(fill_persistent_kernel<NB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)R0Cfg<NB>::SMEM));
    CK(cudaFuncSetAttribute(fill_persistent_kernel<NB>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ctx->persist_occ[NB], fill_persistent_kernel<NB>,
                                                     R0Cfg<NB>::THREADS, R0Cfg<NB>::SMEM));
    if (NB == 8) {
        CK(cudaFuncSetAttribute(r0_wide_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)WideCfg<2>::SMEM));
        CK(cudaFuncSetAttribute(r0_wide_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)WideCfg<3>::SMEM));
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ctx->wide_occ[2], r0_wide_kernel<2>, 128, WideCfg<2>::SMEM));
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ctx->wide_occ[3], r0_wide_kernel<3>, 128, WideCfg<3>::SMEM));
        CK(cudaFuncSetAttribute(r0_large_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)WideShape::SMEM));
        CK(cudaFuncSetAttribute(finalize_wide_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)fin_wide_smem(FIN_WIDE_MAX_NP)));
        CK(cudaFuncSetAttribute(large_tile_local_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)LARGE_LOCAL_SMEM));
    }
    return BPMAX_OK;
}

struct KernelProfile {
    bool on = false;
    cudaEvent_t a = nullptr, b = nullptr;
    float ms[3] = {0, 0, 0};
    long launches[3] = {0, 0, 0};
};

// brackets one launch with events when profiling (eager runs only, never inside a capture)
struct ProfScope {
    bpmax_ctx *ctx;
    KernelProfile *kp;
    int kind;
    ProfScope(bpmax_ctx *c, KernelProfile *k, int kind_) : ctx(c), kp(k), kind(kind_)
    {
        if (kp && kp->on) cudaEventRecord(kp->a, ctx->stream);
    }
    ~ProfScope()
    {
        if (kp && kp->on) {
            cudaEventRecord(kp->b, ctx->stream);
            cudaEventSynchronize(kp->b);
            float t = 0.f;
            cudaEventElapsedTime(&t, kp->a, kp->b);
            kp->ms[kind] += t;
            kp->launches[kind] += 1;
        }
    }
};

int enqueue_fill(bpmax_ctx *ctx, Plan &P, KernelProfile *kp = nullptr)
{
    long launches = 0;
    CK(cudaMemsetAsync(ctx->F.p, 0, (size_t)P.F_floats * sizeof(float), ctx->stream));
    CK(cudaMemsetAsync(ctx->S.p, 0, (size_t)P.S_floats * sizeof(float), ctx->stream));  // S1 starts at 0
    CK(cudaMemsetAsync(ctx->errflag.p, 0, sizeof(int), ctx->stream));
    if (P.r0_only) {
        ProfScope ps(ctx, kp, 0);
        r0only_prep_kernel<<<(int)P.pairs.size(), 256, 0, ctx->stream>>>((const PairDesc *)ctx->pairs.p, (float *)ctx->S.p);
        launches += 1;
    } else {
        ProfScope ps(ctx, kp, 0);
        single_strand_kernel<<<(int)P.pairs.size(), 512, 0, ctx->stream>>>(
            (const PairDesc *)ctx->pairs.p, (const uint8_t *)ctx->bases.p, (float *)ctx->S.p, ctx->W);
        for (int p = 0; p < (int)P.pairs.size(); ++p)  // wider tables: one launch per diagonal of S2
            if (P.pairs[p].Np > WIDE_TILE_MAX_NP)
                for (int d = 4; d < P.pairs[p].N; ++d, ++launches)
                    s2_diag_kernel<<<(P.pairs[p].N - d + 7) / 8, 256, 0, ctx->stream>>>(
                        (const PairDesc *)ctx->pairs.p, p, (const uint8_t *)ctx->bases.p, (float *)ctx->S.p, ctx->W, d);
        s2_aux_kernel<<<(int)P.pairs.size(), 256, 0, ctx->stream>>>((const PairDesc *)ctx->pairs.p, (float *)ctx->S.p);
        launches += 2;
    }
    const bool prof = kp && kp->on;
    if (P.persistent) {  // one persistent launch per width class: side by side on the class streams, or in turn
        const int nclass = (int)P.pclasses.size();
        int *cnt = (int *)ctx->pcnt.p;
        int *diag_done = cnt + 64, *prod_done = diag_done + align64(P.n_counters);
        CK(cudaMemsetAsync(cnt, 0, ((size_t)64 + align64(P.n_counters) + P.prod_need.size()) * sizeof(int), ctx->stream));
        const bool pfork = !prof && nclass > 1 && P.persist == 1;
        if (pfork) {
            CK(cudaEventRecord(ctx->fork_ev, ctx->stream));
            for (int k = 0; k < std::min(nclass, MAX_CLASS_STREAMS); ++k)
                CK(cudaStreamWaitEvent(ctx->class_stream[k], ctx->fork_ev, 0));
        }
        for (int c = 0; c < nclass; ++c, ++launches) {
            const auto &pcl = P.pclasses[c];
            const cudaStream_t st = pfork ? ctx->class_stream[c % MAX_CLASS_STREAMS] : ctx->stream;
            const PersistCtl pctl{(const PItem *)ctx->pq.p + pcl.first, pcl.count, cnt + c, diag_done, prod_done,
                                  (const int *)ctx->pneed.p};
            ProfScope ps(ctx, kp, 1);
            switch (pcl.np / 8) {
            case 1: launch_persist<1>(ctx, pctl, pcl.ctas, st); break;
            case 2: launch_persist<2>(ctx, pctl, pcl.ctas, st); break;
            case 3: launch_persist<3>(ctx, pctl, pcl.ctas, st); break;
            case 4: launch_persist<4>(ctx, pctl, pcl.ctas, st); break;
            case 5: launch_persist<5>(ctx, pctl, pcl.ctas, st); break;
            case 6: launch_persist<6>(ctx, pctl, pcl.ctas, st); break;
            case 7: launch_persist<7>(ctx, pctl, pcl.ctas, st); break;
            default: launch_persist<8>(ctx, pctl, pcl.ctas, st); break;
            }
        }
        if (pfork)
            for (int k = 0; k < std::min(nclass, MAX_CLASS_STREAMS); ++k) {
                CK(cudaEventRecord(ctx->join_ev[k], ctx->class_stream[k]));
                CK(cudaStreamWaitEvent(ctx->stream, ctx->join_ev[k], 0));
            }
        CK(cudaGetLastError());
        P.launches = launches;
        return BPMAX_OK;
    }
    // pairs of different inner widths never interact: each width class runs its own chain of
    // diagonals on its own stream (parallel branches of the captured graph); profiling runs
    // serialise everything on the main stream so every launch can be timed
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(ctx->stream, &cap));
    const bool capturing = cap == cudaStreamCaptureStatusActive;
    const bool fork = !prof && P.classes.size() > 1 && P.class_streams;
    auto chain_of = [&](int np) {
        if (!fork) return 0;
        return (int)(std::find(P.classes.begin(), P.classes.end(), np) - P.classes.begin()) % MAX_CLASS_STREAMS;
    };
    auto stream_of = [&](int np) { return fork ? ctx->class_stream[chain_of(np)] : ctx->stream; };
    const int nstreams = fork ? std::min((int)P.classes.size(), MAX_CLASS_STREAMS) : 0;
    // product launches that read only diagonals <= d-2 (part 0) run on each chain's side stream,
    // after the finalize of d-2, so they overlap the finalize of d-1; the chain's finalize of d
    // waits for them
    bool any_part0 = false;
    for (const auto &L : P.r0_launches) any_part0 = any_part0 || L.part == 0;
    const bool split = !prof && any_part0;
    const int nside = split ? std::max(nstreams, 1) : 0;
    if (fork || split) {
        CK(cudaEventRecord(ctx->fork_ev, ctx->stream));
        for (int k = 0; k < nstreams; ++k) CK(cudaStreamWaitEvent(ctx->class_stream[k], ctx->fork_ev, 0));
        for (int k = 0; k < nside; ++k) CK(cudaStreamWaitEvent(ctx->side_stream[k], ctx->fork_ev, 0));
    }
    bool side_pending[MAX_CLASS_STREAMS] = {};
    size_t ri = 0, fi = 0;
    for (int d = 0; d < P.maxM; ++d) {
        for (; ri < P.r0_launches.size() && P.r0_launches[ri].d == d; ++ri, ++launches) {
            const auto &L = P.r0_launches[ri];
            const int c = chain_of(L.np);
            cudaStream_t st = stream_of(L.np);
            if (split && L.part == 0) {
                // Part 0 of diagonal d (offset pairs >= 1) may run beside the finalize of d-1 because:
                //  1. it reads only tables of diagonals <= d-2, and waits here for the finalize of d-2,
                //     the last writer of those tables and of the SW1 candidates pushed into the still
                //     cleared tables of diagonal d (a finalize of diagonal e writes only the tables of
                //     e, the S1 pieces of e and the pushes into e+2);
                //  2. it writes the tables of diagonal d only through atomicMax of partial maxima,
                //     which commutes with part 1's merges and with those pushes (all values >= +0);
                //  3. the finalize of d-1 writes no table of diagonal d, and the finalize of d waits
                //     for both parts (side_done_ev below).
                // A finalize that wrote diagonal d, or a product merge that was not an atomic max,
                // would race here.
                st = ctx->side_stream[c];
                if (d >= 2) CK(cudaStreamWaitEvent(st, ctx->fin_ev[c][d & 1], 0));  // finalize of d-2
            }
            {
                ProfScope ps(ctx, kp, 1);
                switch (L.np > MAX_SMALL_NP ? 0 : L.np / 8) {
                case 0:
                    if (L.np <= WIDE_TILE_MAX_NP)
                        launch_r0_wide(ctx, P, L, st);
                    else
                        launch_r0_large(ctx, L, st);
                    break;
                case 1: launch_r0<1>(ctx, P, L, st); break;
                case 2: launch_r0<2>(ctx, P, L, st); break;
                case 3: launch_r0<3>(ctx, P, L, st); break;
                case 4: launch_r0<4>(ctx, P, L, st); break;
                case 5: launch_r0<5>(ctx, P, L, st); break;
                case 6: launch_r0<6>(ctx, P, L, st); break;
                case 7: launch_r0<7>(ctx, P, L, st); break;
                default: launch_r0<8>(ctx, P, L, st); break;
                }
            }
            if (split && L.part == 0) {
                CK(cudaEventRecord(ctx->side_done_ev[c], st));
                side_pending[c] = true;
            }
        }
        for (; fi < P.fin_launches.size() && P.fin_launches[fi].d == d; ++fi, ++launches) {
            const auto &L = P.fin_launches[fi];
            const int c = chain_of(L.np);
            const cudaStream_t st = stream_of(L.np);
            if (side_pending[c]) CK(cudaStreamWaitEvent(st, ctx->side_done_ev[c], 0));
            {
                ProfScope ps(ctx, kp, 2);
                if (P.r0_only) {
                    launch_r0only_fin(ctx, L, st);
                } else {
                    switch (L.np > MAX_SMALL_NP ? 0 : L.np / 8) {
                    case 0: launches += launch_fin_large(ctx, L, st) - 1; break;
                    case 1: launch_fin<1>(ctx, L, st); break;
                    case 2: launch_fin<2>(ctx, L, st); break;
                    case 3: launch_fin<3>(ctx, L, st); break;
                    case 4: launch_fin<4>(ctx, L, st); break;
                    case 5: launch_fin<5>(ctx, L, st); break;
                    case 6: launch_fin<6>(ctx, L, st); break;
                    case 7: launch_fin<7>(ctx, L, st); break;
                    default: launch_fin<8>(ctx, L, st); break;
                    }
                }
            }
            if (split) CK(cudaEventRecord(ctx->fin_ev[c][d & 1], st));
        }
        for (bool &p : side_pending) p = false;
        // outer diagonal d is final: rows of the reference layout that end on it can be copied out
        // (events recorded as external nodes of the captured graph; eager runs record none)
        if (!P.diag_ev.empty() && !prof && capturing)
            CK(cudaEventRecordWithFlags(P.diag_ev[d], ctx->stream, cudaEventRecordExternal));
    }
    for (int k = 0; k < nside; ++k) {  // join the side streams back into the main stream
        CK(cudaEventRecord(ctx->side_join_ev[k], ctx->side_stream[k]));
        CK(cudaStreamWaitEvent(ctx->stream, ctx->side_join_ev[k], 0));
    }
    for (int k = 0; k < nstreams; ++k) {  // join the class chains back into the main stream
        CK(cudaEventRecord(ctx->join_ev[k], ctx->class_stream[k]));
        CK(cudaStreamWaitEvent(ctx->stream, ctx->join_ev[k], 0));
    }
    CK(cudaGetLastError());
    P.launches = launches;
    return BPMAX_OK;
}

// Makes the plan for these shapes current (reusing the cached one and its graph when the
// shapes repeat) and uploads the sequences. Sequences are validated by the caller.
int prepare(bpmax_ctx *ctx, const std::vector<int> &Ms, const std::vector<int> &Ns,
            const std::vector<const int *> &s1s, const std::vector<const int *> &s2s)
{
    int st;
    const auto tu = ctx->tuned.find(shape_key(Ms, Ns));
    const Tuned want = tu != ctx->tuned.end() ? tu->second
                                              : Tuned{ctx->r0_pairs_per_job, ctx->r0_merge_items, ctx->class_streams,
                                                      ctx->r0_variant, ctx->wide_stages, ctx->class_share, ctx->persist};
    const bool same_tuning = ctx->plan.pairs_per_job == want[0] && ctx->plan.merge_items == want[1] &&
                             ctx->plan.class_streams == want[2] && ctx->plan.r0_variant == want[3] &&
                             ctx->plan.wide_stages == want[4] && ctx->plan.class_share == want[5] &&
                             ctx->plan.persist == want[6] && ctx->plan.copyout == ctx->copyout &&
                             ctx->plan.ref.out == ctx->want_ref.out && ctx->plan.ref.T == ctx->want_ref.T &&
                             ctx->plan.ref.Ns == ctx->want_ref.Ns;
    if (!(ctx->plan_valid && ctx->plan.Ms == Ms && ctx->plan.Ns == Ns && same_tuning && ctx->plan.r0_only == ctx->r0_only &&
          ctx->plan.split == ctx->allow_split)) {
        if (ctx->plan.graph) cudaGraphExecDestroy(ctx->plan.graph);
        ctx->plan.graph = nullptr;
        for (cudaEvent_t e : ctx->plan.diag_ev) cudaEventDestroy(e);
        ctx->plan.diag_ev.clear();
        ctx->plan_valid = false;
        if ((st = build_plan(ctx, Ms, Ns, ctx->plan)) != BPMAX_OK) return st;
        Plan &P = ctx->plan;
        P.r0_only = ctx->r0_only;
        P.ref = ctx->want_ref;
        if (P.pairs.size() == 1) {
            P.diag_ev.assign(P.maxM, nullptr);
            for (auto &e : P.diag_ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        }
        if ((st = ensure(ctx, ctx->F, P.F_floats * sizeof(float))) != BPMAX_OK) return st;
        if (P.any_large && (st = ensure(ctx, ctx->FT, P.F_floats * sizeof(float))) != BPMAX_OK) return st;
        if ((st = ensure(ctx, ctx->errflag, sizeof(int))) != BPMAX_OK) return st;
        if ((st = ensure(ctx, ctx->S, P.S_floats * sizeof(float))) != BPMAX_OK) return st;
        if ((st = ensure(ctx, ctx->bases, P.bases_bytes + 16)) != BPMAX_OK) return st;
        if ((st = ensure(ctx, ctx->pairs, P.pairs.size() * sizeof(PairDesc))) != BPMAX_OK) return st;
        if ((st = ensure(ctx, ctx->r0jobs, P.r0_jobs.size() * sizeof(R0Job))) != BPMAX_OK) return st;
        if ((st = ensure(ctx, ctx->r0ljobs, P.r0l_jobs.size() * sizeof(R0JobL))) != BPMAX_OK) return st;
        if ((st = ensure(ctx, ctx->r0wjobs, P.r0w_jobs.size() * sizeof(R0JobW))) != BPMAX_OK) return st;
        if (P.persistent) {
            if ((st = ensure(ctx, ctx->pq, P.pitems.size() * sizeof(PItem))) != BPMAX_OK) return st;
            if ((st = ensure(ctx, ctx->pneed, P.prod_need.size() * sizeof(int))) != BPMAX_OK) return st;
            if ((st = ensure(ctx, ctx->pcnt, (64 + align64(P.n_counters) + P.prod_need.size()) * sizeof(int))) != BPMAX_OK)
                return st;
            CK(cudaMemcpyAsync(ctx->pq.p, P.pitems.data(), P.pitems.size() * sizeof(PItem), cudaMemcpyHostToDevice,
                               ctx->stream));
            CK(cudaMemcpyAsync(ctx->pneed.p, P.prod_need.data(), P.prod_need.size() * sizeof(int),
                               cudaMemcpyHostToDevice, ctx->stream));
        }
        if ((st = ensure(ctx, ctx->celljobs, P.cell_jobs.size() * sizeof(CellJob))) != BPMAX_OK) return st;
        if ((st = ensure(ctx, ctx->scores, P.pairs.size() * sizeof(float))) != BPMAX_OK) return st;
        CK(cudaMemcpyAsync(ctx->pairs.p, P.pairs.data(), P.pairs.size() * sizeof(PairDesc), cudaMemcpyHostToDevice, ctx->stream));
        if (!P.r0_jobs.empty())
            CK(cudaMemcpyAsync(ctx->r0jobs.p, P.r0_jobs.data(), P.r0_jobs.size() * sizeof(R0Job), cudaMemcpyHostToDevice, ctx->stream));
        if (!P.r0w_jobs.empty())
            CK(cudaMemcpyAsync(ctx->r0wjobs.p, P.r0w_jobs.data(), P.r0w_jobs.size() * sizeof(R0JobW), cudaMemcpyHostToDevice,
                               ctx->stream));
        if (!P.r0l_jobs.empty())
            CK(cudaMemcpyAsync(ctx->r0ljobs.p, P.r0l_jobs.data(), P.r0l_jobs.size() * sizeof(R0JobL), cudaMemcpyHostToDevice,
                               ctx->stream));
        CK(cudaMemcpyAsync(ctx->celljobs.p, P.cell_jobs.data(), P.cell_jobs.size() * sizeof(CellJob), cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        ctx->plan_valid = true;
    }
    Plan &P = ctx->plan;
    if (P.r0_only) {  // the sequences are the base values themselves: seq1, then seq2 unreversed
        std::vector<float> hv;
        for (int i = 0; i < Ms[0]; ++i) hv.push_back((float)s1s[0][i]);
        for (int i = 0; i < Ns[0]; ++i) hv.push_back((float)s2s[0][i]);
        if ((st = ensure(ctx, ctx->r0vals, hv.size() * sizeof(float))) != BPMAX_OK) return st;
        CK(cudaMemcpyAsync(ctx->r0vals.p, hv.data(), hv.size() * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        return BPMAX_OK;
    }
    // sequences: seq1 as is, seq2 reversed (V3/transform_reverse_1D_to_2D.c:131-135)
    std::vector<uint8_t> hb(P.bases_bytes);
    for (size_t p = 0; p < P.pairs.size(); ++p) {
        const PairDesc &pd = P.pairs[p];
        for (int i = 0; i < pd.M; ++i) hb[pd.seq1_off + i] = (uint8_t)s1s[p][i];
        for (int i = 0; i < pd.N; ++i) hb[pd.seq2_off + i] = (uint8_t)s2s[p][pd.N - 1 - i];
    }
    CK(cudaMemcpyAsync(ctx->bases.p, hb.data(), hb.size(), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return BPMAX_OK;
}

// Launches the fill of the current plan (graph captured on first use) on the context's stream.
int launch_fill(bpmax_ctx *ctx)
{
    Plan &P = ctx->plan;
    int st;
    if (ctx->inject_wait_timeout) {  // test of the timeout path: one eager run, outside the graph
        CK(cudaEventRecord(ctx->ev0, ctx->stream));
        if ((st = enqueue_fill(ctx, P)) != BPMAX_OK) return st;
        for (cudaEvent_t e : P.diag_ev) CK(cudaEventRecord(e, ctx->stream));  // copy-out waits for the whole fill
        CK(cudaEventRecord(ctx->ev1, ctx->stream));
        gather_scores_kernel<<<((int)P.pairs.size() + 127) / 128, 128, 0, ctx->stream>>>(
            (const PairDesc *)ctx->pairs.p, (const float *)ctx->F.p, (int)P.pairs.size(), (float *)ctx->scores.p);
        CK(cudaGetLastError());
        return BPMAX_OK;
    }
    if (!P.graph) {
        cudaGraph_t g;
        CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        st = enqueue_fill(ctx, P);
        cudaGraph_t captured = nullptr;
        cudaError_t ce = cudaStreamEndCapture(ctx->stream, &captured);
        if (st != BPMAX_OK) {
            if (captured) cudaGraphDestroy(captured);
            return st;
        }
        if (ce != cudaSuccess) return fail(ctx, BPMAX_ECUDA, "graph capture: %s", cudaGetErrorString(ce));
        g = captured;
        CK(cudaGraphInstantiate(&P.graph, g, 0));
        cudaGraphDestroy(g);
    }
    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    CK(cudaGraphLaunch(P.graph, ctx->stream));
    CK(cudaEventRecord(ctx->ev1, ctx->stream));
    gather_scores_kernel<<<((int)P.pairs.size() + 127) / 128, 128, 0, ctx->stream>>>(
        (const PairDesc *)ctx->pairs.p, (const float *)ctx->F.p, (int)P.pairs.size(), (float *)ctx->scores.p);
    CK(cudaGetLastError());
    return BPMAX_OK;
}

// Waits for the fill launched by launch_fill, reads its error word and times it.
int finish_fill(bpmax_ctx *ctx)
{
    Plan &P = ctx->plan;
    int errv = 0;
    CK(cudaMemcpyAsync(&errv, ctx->errflag.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaEventSynchronize(ctx->ev1));
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaEventElapsedTime(&ctx->last_ms, ctx->ev0, ctx->ev1));
    ctx->last_launches = P.launches + 1;  // + the score gather
    const bool injected = ctx->inject_wait_timeout;
    ctx->inject_wait_timeout = false;  // one-shot
    if (errv)
        return fail(ctx, BPMAX_ETIMEOUT, "a product kernel gave up waiting for its operand copies%s",
                    injected ? " (test mode: no copies were issued)" : "");
    return BPMAX_OK;
}

int run_fill(bpmax_ctx *ctx)
{
    const int st = launch_fill(ctx);
    return st ? st : finish_fill(ctx);
}

int check_pair(bpmax_ctx *ctx, const int *s1, long M, const int *s2, long N)
{
    if (!s1 || !s2) return fail(ctx, BPMAX_EINVAL, "null sequence pointer");
    if (M < 1 || N < 1) return fail(ctx, BPMAX_EINVAL, "sequence lengths must be >= 1 (M=%ld, N=%ld)", M, N);
    if (M > 65535 || N > MAX_NP) return fail(ctx, BPMAX_EINVAL, "sequence length too large (M=%ld, N=%ld)", M, N);
    for (long i = 0; i < M; ++i)
        if (s1[i] < 0 || s1[i] > 4) return fail(ctx, BPMAX_EINVAL, "seq1[%ld]=%d is not a base code 0..4", i, s1[i]);
    for (long i = 0; i < N; ++i)
        if (s2[i] < 0 || s2[i] > 4) return fail(ctx, BPMAX_EINVAL, "seq2[%ld]=%d is not a base code 0..4", i, s2[i]);
    return BPMAX_OK;
}

int fill_pairs(bpmax_ctx *ctx, int num_pairs, const int *const *seq1s, const long *Ms, const int *const *seq2s,
               const long *Ns, bool async = false)
{
    if (!ctx) return BPMAX_EINVAL;
    if (num_pairs < 1 || !seq1s || !seq2s || !Ms || !Ns) return fail(ctx, BPMAX_EINVAL, "empty batch");
    std::vector<int> vm(num_pairs), vn(num_pairs);
    std::vector<const int *> a(num_pairs), b(num_pairs);
    for (int p = 0; p < num_pairs; ++p) {
        int st = check_pair(ctx, seq1s[p], Ms[p], seq2s[p], Ns[p]);
        if (st) return st;
        vm[p] = (int)Ms[p];
        vn[p] = (int)Ns[p];
        a[p] = seq1s[p];
        b[p] = seq2s[p];
    }
    CK(cudaSetDevice(ctx->device));
    int st = prepare(ctx, vm, vn, a, b);
    if (st) return st;
    return async ? launch_fill(ctx) : run_fill(ctx);
}

int ensure_host_stage(bpmax_ctx *ctx, size_t bytes)
{
    if (ctx->host_stage_bytes >= bytes) return BPMAX_OK;
    for (int i = 0; i < 2; ++i) {
        if (ctx->host_stage[i]) cudaFreeHost(ctx->host_stage[i]);
        ctx->host_stage[i] = nullptr;
    }
    ctx->host_stage_bytes = 0;
    for (int i = 0; i < 2; ++i) CK(cudaMallocHost(&ctx->host_stage[i], bytes));
    ctx->host_stage_bytes = bytes;
    return BPMAX_OK;
}

bool is_pinned(const void *p)
{
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeHost;
}

}  // namespace

extern "C" {

const char *bpmax_gpu_status_string(int s)
{
    switch (s) {
    case BPMAX_OK: return "ok";
    case BPMAX_EINVAL: return "invalid argument";
    case BPMAX_ENOMEM: return "out of memory";
    case BPMAX_ECUDA: return "CUDA error";
    case BPMAX_ENODEV: return "no usable CUDA device";
    case BPMAX_ETIMEOUT: return "device wait timed out";
    default: return "unknown status";
    }
}

int bpmax_gpu_create(int device, bpmax_ctx **out)
{
    if (!out) return BPMAX_EINVAL;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
        cudaGetLastError();
        return BPMAX_ENODEV;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10) {
        cudaGetLastError();
        return BPMAX_ENODEV;  // the kernels are built for sm_100a only
    }
    bpmax_ctx *ctx = new bpmax_ctx();
    ctx->device = device;
    ctx->sms = prop.multiProcessorCount;
    const float ref_w[12] = {1.0f, 1.0f, 3.0f, 3.0f, 1.5f, 1.5f, 1.0f, 1.0f, 3.0f, 3.0f, 1.5f, 1.5f};
    memcpy(ctx->W.w, ref_w, sizeof ref_w);
    int st = BPMAX_OK;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&ctx->ev0) != cudaSuccess || cudaEventCreate(&ctx->ev1) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->stage_ev[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->stage_ev[1], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->fork_ev, cudaEventDisableTiming) != cudaSuccess)
        st = BPMAX_ECUDA;
    if (st == BPMAX_OK && cudaStreamCreateWithFlags(&ctx->aux_stream, cudaStreamNonBlocking) != cudaSuccess) st = BPMAX_ECUDA;
    for (int k = 0; k < MAX_CLASS_STREAMS && st == BPMAX_OK; ++k)
        if (cudaStreamCreateWithFlags(&ctx->class_stream[k], cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&ctx->join_ev[k], cudaEventDisableTiming) != cudaSuccess ||
            cudaStreamCreateWithFlags(&ctx->side_stream[k], cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&ctx->side_done_ev[k], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&ctx->side_join_ev[k], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&ctx->fin_ev[k][0], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&ctx->fin_ev[k][1], cudaEventDisableTiming) != cudaSuccess)
            st = BPMAX_ECUDA;
    if (st == BPMAX_OK) st = set_smem_attr<1>(ctx);
    if (st == BPMAX_OK) st = set_smem_attr<2>(ctx);
    if (st == BPMAX_OK) st = set_smem_attr<3>(ctx);
    if (st == BPMAX_OK) st = set_smem_attr<4>(ctx);
    if (st == BPMAX_OK) st = set_smem_attr<5>(ctx);
    if (st == BPMAX_OK) st = set_smem_attr<6>(ctx);
    if (st == BPMAX_OK) st = set_smem_attr<7>(ctx);
    if (st == BPMAX_OK) st = set_smem_attr<8>(ctx);
    if (st != BPMAX_OK) {
        cudaGetLastError();
        bpmax_gpu_destroy(ctx);
        return st;
    }
    *out = ctx;
    return BPMAX_OK;
}

void bpmax_gpu_destroy(bpmax_ctx *ctx)
{
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->plan.graph) cudaGraphExecDestroy(ctx->plan.graph);
    for (DevBuf *b : {&ctx->tbstack, &ctx->grads, &ctx->tbstatus, &ctx->F, &ctx->FT, &ctx->S, &ctx->bases, &ctx->pairs,
                      &ctx->r0jobs, &ctx->r0ljobs, &ctx->r0wjobs, &ctx->pq, &ctx->pcnt, &ctx->pneed, &ctx->celljobs,
                      &ctx->scores, &ctx->conv, &ctx->refdev, &ctx->errflag,
                      &ctx->r0vals})
        if (b->p) cudaFree(b->p);
    for (int i = 0; i < 2; ++i) {
        if (ctx->host_stage[i]) cudaFreeHost(ctx->host_stage[i]);
        if (ctx->stage_ev[i]) cudaEventDestroy(ctx->stage_ev[i]);
    }
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->fork_ev) cudaEventDestroy(ctx->fork_ev);
    for (cudaEvent_t e : ctx->plan.diag_ev) cudaEventDestroy(e);
    if (ctx->aux_stream) cudaStreamDestroy(ctx->aux_stream);
    for (int k = 0; k < MAX_CLASS_STREAMS; ++k) {
        if (ctx->class_stream[k]) cudaStreamDestroy(ctx->class_stream[k]);
        if (ctx->join_ev[k]) cudaEventDestroy(ctx->join_ev[k]);
        if (ctx->side_stream[k]) cudaStreamDestroy(ctx->side_stream[k]);
        for (cudaEvent_t e : {ctx->side_done_ev[k], ctx->side_join_ev[k], ctx->fin_ev[k][0], ctx->fin_ev[k][1]})
            if (e) cudaEventDestroy(e);
    }
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char *bpmax_gpu_last_error(const bpmax_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int bpmax_gpu_set_weights(bpmax_ctx *ctx, const float *w)
{
    if (!ctx) return BPMAX_EINVAL;
    if (!w || !weights_ok(w)) return fail(ctx, BPMAX_EINVAL, "weights must be 12 finite values >= +0");
    memcpy(ctx->W.w, w, sizeof ctx->W.w);
    // weights are kernel arguments baked into the captured graph: recapture on next use
    if (ctx->plan.graph) {
        cudaGraphExecDestroy(ctx->plan.graph);
        ctx->plan.graph = nullptr;
    }
    return BPMAX_OK;
}

int bpmax_gpu_score(bpmax_ctx *ctx, const int *seq1, long M, const int *seq2, long N, float *score)
{
    if (!ctx) return BPMAX_EINVAL;
    int st = fill_pairs(ctx, 1, &seq1, &M, &seq2, &N);
    if (st) return st;
    if (score) CK(cudaMemcpy(score, ctx->scores.p, sizeof(float), cudaMemcpyDeviceToHost));
    return BPMAX_OK;
}

int bpmax_gpu_score_batch(bpmax_ctx *ctx, int num_pairs, const int *const *seq1s, const long *Ms,
                          const int *const *seq2s, const long *Ns, float *scores)
{
    if (!ctx) return BPMAX_EINVAL;
    int st = fill_pairs(ctx, num_pairs, seq1s, Ms, seq2s, Ns);
    if (st) return st;
    if (scores) CK(cudaMemcpy(scores, ctx->scores.p, num_pairs * sizeof(float), cudaMemcpyDeviceToHost));
    return BPMAX_OK;
}

int bpmax_gpu_score_each(bpmax_ctx *ctx, int num_pairs, const int *const *seq1s, const long *Ms,
                         const int *const *seq2s, const long *Ns, float *scores)
{
    if (!ctx) return BPMAX_EINVAL;
    if (num_pairs < 1) return fail(ctx, BPMAX_EINVAL, "empty batch");
    float total = 0.f;
    long launches = 0;
    for (int p = 0; p < num_pairs; ++p) {
        int st = fill_pairs(ctx, 1, seq1s + p, Ms + p, seq2s + p, Ns + p);
        if (st) return st;
        total += ctx->last_ms;
        launches += ctx->last_launches;
        if (scores) CK(cudaMemcpy(scores + p, ctx->scores.p, sizeof(float), cudaMemcpyDeviceToHost));
    }
    ctx->last_ms = total;
    ctx->last_launches = launches;
    return BPMAX_OK;
}

int bpmax_gpu_r0_only(bpmax_ctx *ctx, const int *seq1, long M, const int *seq2, long N, float *F_compact,
                      float *score)
{
    if (!ctx) return BPMAX_EINVAL;
    if (!seq1 || !seq2) return fail(ctx, BPMAX_EINVAL, "null sequence");
    // the reference's domain {M,N | M>=2 && N>=2} (IPDPSW/.../ospsq_float.ab:1)
    if (M < 2 || N < 2 || M > 65535) return fail(ctx, BPMAX_EINVAL, "The value of parameters are not valid.");
    if (padded_width((int)N) > MAX_NP) return fail(ctx, BPMAX_EINVAL, "strand-2 length %ld > %d is not supported", N, MAX_NP);
    for (long i = 0; i < M; ++i)
        if (seq1[i] < 0) return fail(ctx, BPMAX_EINVAL, "seq1[%ld] = %d < 0: values must be non-negative", i, seq1[i]);
    for (long i = 0; i < N; ++i)
        if (seq2[i] < 0) return fail(ctx, BPMAX_EINVAL, "seq2[%ld] = %d < 0: values must be non-negative", i, seq2[i]);
    CK(cudaSetDevice(ctx->device));
    ctx->r0_only = true;
    int st = prepare(ctx, {(int)M}, {(int)N}, {seq1}, {seq2});
    ctx->r0_only = false;
    if (st) return st;
    if ((st = run_fill(ctx)) != BPMAX_OK) return st;
    if (score) CK(cudaMemcpy(score, ctx->scores.p, sizeof(float), cudaMemcpyDeviceToHost));
    if (!F_compact) return BPMAX_OK;
    const long long n_out = M * (M + 1) / 2 * N * N;
    if ((st = ensure(ctx, ctx->conv, n_out * sizeof(float))) != BPMAX_OK) return st;
    to_compact_kernel<<<4 * ctx->sms, 256, 0, ctx->stream>>>((const PairDesc *)ctx->pairs.p, (const float *)ctx->F.p,
                                                             n_out, (float *)ctx->conv.p);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(F_compact, ctx->conv.p, n_out * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return BPMAX_OK;
}

int bpmax_gpu_fill_compact(bpmax_ctx *ctx, const int *seq1, long M, const int *seq2, long N, float *F_compact,
                           float *score)
{
    if (!ctx) return BPMAX_EINVAL;
    int st = fill_pairs(ctx, 1, &seq1, &M, &seq2, &N);
    if (st) return st;
    if (score) CK(cudaMemcpy(score, ctx->scores.p, sizeof(float), cudaMemcpyDeviceToHost));
    if (!F_compact) return BPMAX_OK;
    const long long n_out = M * (M + 1) / 2 * N * N;
    if ((st = ensure(ctx, ctx->conv, n_out * sizeof(float))) != BPMAX_OK) return st;
    to_compact_kernel<<<4 * ctx->sms, 256, 0, ctx->stream>>>((const PairDesc *)ctx->pairs.p, (const float *)ctx->F.p,
                                                             n_out, (float *)ctx->conv.p);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(F_compact, ctx->conv.p, n_out * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return BPMAX_OK;
}

int bpmax_gpu_fill(bpmax_ctx *ctx, const int *seq1, long M, const int *seq2, long N, long N_tile, float *F_lin,
                   float *score)
{
    if (!ctx) return BPMAX_EINVAL;
    // preconditions of V3/bpmax.c:131 (N_sec>=2 and 0<=R<N_tile follow from the layout)
    if (M < 1 || N < 8 || N_tile < 4) return fail(ctx, BPMAX_EINVAL, "The value of parameters are not valid.");
    const long Ns = (N + N_tile - 1) / N_tile;
    if (Ns < 2) return fail(ctx, BPMAX_EINVAL, "The value of parameters are not valid. (N_sec=%ld < 2)", Ns);
    if (!F_lin) {
        int st = fill_pairs(ctx, 1, &seq1, &M, &seq2, &N);
        if (st) return st;
        if (score) CK(cudaMemcpy(score, ctx->scores.p, sizeof(float), cudaMemcpyDeviceToHost));
        return BPMAX_OK;
    }
    const long long cell_f = (long long)Ns * Ns * (N_tile + 1) * N_tile;
    // The table is copied out while the fill still runs (aux stream, waiting on the per-diagonal
    // events the graph records). Into pinned memory: per outer diagonal, as soon as it is final --
    // its cells (i1, i1+d) lie (M+1) cells apart in the reference layout, so one strided copy
    // places a diagonal converted into a staging slot, and the copy-out ends one diagonal after the
    // fill. Into pageable memory (through a pinned staging buffer and a host copy): per outer row,
    // contiguous in the layout and final once outer diagonal M-1-i1 is, from the last one up.
    const long long row_max = (long long)M * cell_f;
    int st;
    if ((st = ensure(ctx, ctx->conv, 2 * row_max * sizeof(float))) != BPMAX_OK) return st;
    const bool pinned = is_pinned(F_lin);
    if (!pinned && (st = ensure_host_stage(ctx, row_max * sizeof(float))) != BPMAX_OK) return st;
    // Widths <= 64 into pinned memory: the finalize launches themselves write every cell they
    // complete in the reference layout (diagonal-major, on the device), so only copy engines work
    // beside the fill, which keeps its split schedule. Without room for that buffer, or wider,
    // a conversion launch per diagonal does it (those launches share the SMs with the fill's,
    // so the fill then runs unsplit).
    const size_t fused_bytes = (size_t)(M * (M + 1) / 2) * cell_f * sizeof(float);
    bool fused = false;
    if (pinned && padded_width((int)N) <= MAX_SMALL_NP) {
        fused = ctx->refdev.bytes >= fused_bytes;
        if (!fused) {
            if (ctx->refdev.p) cudaFree(ctx->refdev.p);
            ctx->refdev = DevBuf{};
            void *p = nullptr;
            if (cudaMalloc(&p, fused_bytes) == cudaSuccess) {
                ctx->refdev = DevBuf{p, fused_bytes};
                fused = true;
            } else {
                cudaGetLastError();  // out of memory: not sticky, take the conversion launches
            }
        }
    }
    ctx->want_ref = fused ? RefOut{(float *)ctx->refdev.p, (int)N_tile, (int)Ns} : RefOut{nullptr, 0, 0};
    ctx->allow_split = fused;
    ctx->copyout = true;
    st = fill_pairs(ctx, 1, &seq1, &M, &seq2, &N, true);
    ctx->allow_split = true;
    ctx->copyout = false;
    ctx->want_ref = RefOut{nullptr, 0, 0};
    if (st != BPMAX_OK) return st;
    const std::vector<cudaEvent_t> &dev = ctx->plan.diag_ev;
    if (fused) {
        const size_t cell_b = (size_t)cell_f * sizeof(float);
        for (long d = 0; d < M; ++d) {
            const float *src = (const float *)ctx->refdev.p + (d * M - d * (d - 1) / 2) * cell_f;
            CK(cudaStreamWaitEvent(ctx->aux_stream, dev[d], 0));
            CK(cudaMemcpy2DAsync(F_lin + d * cell_f, (size_t)(M + 1) * cell_b, src, cell_b, cell_b, (size_t)(M - d),
                                 cudaMemcpyDeviceToHost, ctx->aux_stream));
        }
        CK(cudaStreamSynchronize(ctx->aux_stream));
        if ((st = finish_fill(ctx)) != BPMAX_OK) return st;
        if (score) CK(cudaMemcpy(score, ctx->scores.p, sizeof(float), cudaMemcpyDeviceToHost));
        return BPMAX_OK;
    }
    if (pinned) {
        const size_t cell_b = (size_t)cell_f * sizeof(float);
        for (long d = 0; d < M; ++d) {
            float *slot = (float *)ctx->conv.p + (d & 1) * row_max;
            const long long n_out = (M - d) * cell_f;
            CK(cudaStreamWaitEvent(ctx->aux_stream, dev[d], 0));
            to_reference_diag_kernel<<<(int)std::min<long long>(4 * ctx->sms, (n_out + 255) / 256), 256, 0,
                                       ctx->aux_stream>>>((const PairDesc *)ctx->pairs.p, (const float *)ctx->F.p,
                                                          (int)N_tile, (int)Ns, (int)d, n_out, slot);
            CK(cudaGetLastError());
            CK(cudaMemcpy2DAsync(F_lin + d * cell_f, (size_t)(M + 1) * cell_b, slot, cell_b, cell_b, (size_t)(M - d),
                                 cudaMemcpyDeviceToHost, ctx->aux_stream));
        }
        CK(cudaStreamSynchronize(ctx->aux_stream));
        if ((st = finish_fill(ctx)) != BPMAX_OK) return st;
        if (score) CK(cudaMemcpy(score, ctx->scores.p, sizeof(float), cudaMemcpyDeviceToHost));
        return BPMAX_OK;
    }
    std::vector<long long> pending_n(2, 0);
    std::vector<float *> pending_dst(2, nullptr);
    for (long i1 = M - 1; i1 >= 0; --i1) {
        const int slot = (int)(i1 & 1);
        float *dbuf = (float *)ctx->conv.p + slot * row_max;
        const long long n_out = (M - i1) * cell_f;
        float *dst = F_lin + (i1 * M + i1) * cell_f;
        if (pending_dst[slot]) {  // drain the staging buffer this slot used before
            CK(cudaEventSynchronize(ctx->stage_ev[slot]));
            memcpy(pending_dst[slot], ctx->host_stage[slot], pending_n[slot] * sizeof(float));
            pending_dst[slot] = nullptr;
        }
        CK(cudaStreamWaitEvent(ctx->aux_stream, dev[M - 1 - i1], 0));
        to_reference_row_kernel<<<4 * ctx->sms, 256, 0, ctx->aux_stream>>>(
            (const PairDesc *)ctx->pairs.p, (const float *)ctx->F.p, (int)N_tile, (int)Ns, (int)i1, n_out, dbuf);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(ctx->host_stage[slot], dbuf, n_out * sizeof(float), cudaMemcpyDeviceToHost, ctx->aux_stream));
        CK(cudaEventRecord(ctx->stage_ev[slot], ctx->aux_stream));
        pending_dst[slot] = dst;
        pending_n[slot] = n_out;
    }
    for (int slot = 0; slot < 2; ++slot)
        if (pending_dst[slot]) {
            CK(cudaEventSynchronize(ctx->stage_ev[slot]));
            memcpy(pending_dst[slot], ctx->host_stage[slot], pending_n[slot] * sizeof(float));
        }
    CK(cudaStreamSynchronize(ctx->aux_stream));
    if ((st = finish_fill(ctx)) != BPMAX_OK) return st;
    if (score) CK(cudaMemcpy(score, ctx->scores.p, sizeof(float), cudaMemcpyDeviceToHost));
    return BPMAX_OK;
}

int bpmax_gpu_grad_batch(bpmax_ctx *ctx, int num_pairs, const int *const *seq1s, const long *Ms,
                         const int *const *seq2s, const long *Ns, float *scores, float *grads)
{
    if (!ctx) return BPMAX_EINVAL;
    int st = fill_pairs(ctx, num_pairs, seq1s, Ms, seq2s, Ns);
    if (st) return st;
    long maxlen = 0;
    for (int p = 0; p < num_pairs; ++p) maxlen = std::max(maxlen, Ms[p] + Ns[p]);
    const int cap = (int)(2 * maxlen + 64);  // DFS depth of the argmax tree <= M + N + 1
    if ((st = ensure(ctx, ctx->tbstack, (size_t)num_pairs * cap * sizeof(TbNode))) != BPMAX_OK) return st;
    if ((st = ensure(ctx, ctx->grads, (size_t)num_pairs * 12 * sizeof(float))) != BPMAX_OK) return st;
    if ((st = ensure(ctx, ctx->tbstatus, (size_t)num_pairs * sizeof(int))) != BPMAX_OK) return st;
    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    traceback_kernel<<<num_pairs, TB_THREADS, 0, ctx->stream>>>(
        (const PairDesc *)ctx->pairs.p, (const float *)ctx->F.p, (const float *)ctx->S.p, (const uint8_t *)ctx->bases.p,
        ctx->W, (TbNode *)ctx->tbstack.p, cap, (float *)ctx->grads.p, (int *)ctx->tbstatus.p);
    CK(cudaGetLastError());
    CK(cudaEventRecord(ctx->ev1, ctx->stream));
    std::vector<int> stat(num_pairs);
    CK(cudaMemcpyAsync(stat.data(), ctx->tbstatus.p, num_pairs * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    if (scores) CK(cudaMemcpyAsync(scores, ctx->scores.p, num_pairs * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    if (grads) CK(cudaMemcpyAsync(grads, ctx->grads.p, num_pairs * 12 * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    float tb_ms = 0.f;
    CK(cudaEventElapsedTime(&tb_ms, ctx->ev0, ctx->ev1));
    ctx->last_ms += tb_ms;
    ctx->last_launches += 1;
    for (int p = 0; p < num_pairs; ++p)
        if (stat[p]) return fail(ctx, BPMAX_ECUDA, "adjoint pass of pair %d stopped (status %d)", p, stat[p]);
    return BPMAX_OK;
}

int bpmax_gpu_profile_kernels(bpmax_ctx *ctx, float *ms, long *launches, double *terms)
{
    if (!ctx) return BPMAX_EINVAL;
    if (!ctx->plan_valid) return fail(ctx, BPMAX_EINVAL, "no fill has run on this context");
    CK(cudaSetDevice(ctx->device));
    KernelProfile kp;
    kp.on = true;
    CK(cudaEventCreate(&kp.a));
    CK(cudaEventCreate(&kp.b));
    int st = enqueue_fill(ctx, ctx->plan, &kp);
    cudaEventDestroy(kp.a);
    cudaEventDestroy(kp.b);
    if (st) return st;
    CK(cudaStreamSynchronize(ctx->stream));
    // algorithmic candidates per kind
    auto C = [](double n) { return n * (n * n - 1) / 6.0; };
    auto T = [](double n) { return n * (n + 1) / 2.0; };
    double t[3] = {0, 0, 0};
    for (const PairDesc &pd : ctx->plan.pairs) {
        if (ctx->plan.r0_only) {  // the double max-plus alone; the other kinds only place values
            t[1] += C(pd.M) * C(pd.N);
            continue;
        }
        t[0] += C(pd.M) + C(pd.N);
        t[1] += C(pd.M) * (C(pd.N) + 2 * T(pd.N));
        t[2] += 2 * T(pd.M) * C(pd.N);
    }
    for (int k = 0; k < 3; ++k) {
        if (ms) ms[k] = kp.ms[k];
        if (launches) launches[k] = kp.launches[k];
        if (terms) terms[k] = t[k];
    }
    return BPMAX_OK;
}

int bpmax_gpu_maxplus_peak(bpmax_ctx *ctx, double *terms_per_s)
{
    if (!ctx || !terms_per_s) return BPMAX_EINVAL;
    CK(cudaSetDevice(ctx->device));
    float *buf = nullptr;
    const int grid = ctx->sms * 8, block = 128, reps = 250;
    CK(cudaMalloc(&buf, (size_t)grid * block * sizeof(float) + 64 * sizeof(float)));
    std::vector<float> h(64);
    for (int i = 0; i < 64; ++i) h[i] = (float)(i % 17);
    cudaMemcpyAsync(buf, h.data(), 64 * sizeof(float), cudaMemcpyHostToDevice, ctx->stream);
    maxplus_peak_kernel<<<grid, block, 0, ctx->stream>>>(buf, buf + 64, reps);
    cudaEventRecord(ctx->ev0, ctx->stream);
    for (int i = 0; i < 3; ++i) maxplus_peak_kernel<<<grid, block, 0, ctx->stream>>>(buf, buf + 64, reps);
    cudaEventRecord(ctx->ev1, ctx->stream);
    cudaError_t e = cudaEventSynchronize(ctx->ev1);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    cudaFree(buf);
    if (e != cudaSuccess) return fail(ctx, BPMAX_ECUDA, "peak probe: %s", cudaGetErrorString(e));
    *terms_per_s = 3.0 * grid * block * (double)reps * (8.0 * MAXPLUS_PEAK_CHAINS) / (ms * 1e-3);
    return BPMAX_OK;
}

int bpmax_gpu_set_tuning(bpmax_ctx *ctx, int key, long value)
{
    if (!ctx) return BPMAX_EINVAL;
    switch (key) {
    case BPMAX_TUNE_R0_PAIRS_PER_JOB:
        if (value < 1) return fail(ctx, BPMAX_EINVAL, "pairs per job must be >= 1");
        ctx->r0_pairs_per_job = (int)std::min<long>(value, 1 << 20);
        break;
    case BPMAX_TUNE_R0_MERGE_ITEMS:
        if (value < 0 || value > 1 << 20) return fail(ctx, BPMAX_EINVAL, "merge cost out of range");
        ctx->r0_merge_items = (int)value;
        break;
    case BPMAX_TUNE_CLASS_STREAMS:
        ctx->class_streams = value != 0;
        break;
    case BPMAX_TUNE_WAIT_LIMIT_US:
        if (value < 1 || value > 600000000L) return fail(ctx, BPMAX_EINVAL, "wait limit out of range (1 us .. 600 s)");
        ctx->wait_ns = (unsigned long long)value * 1000ULL;
        if (ctx->plan.graph) {  // a kernel argument baked into the captured graph: recapture on next use
            cudaGraphExecDestroy(ctx->plan.graph);
            ctx->plan.graph = nullptr;
        }
        break;
    case BPMAX_TUNE_INJECT_WAIT_TIMEOUT:
        ctx->inject_wait_timeout = value != 0;
        break;
    case BPMAX_TUNE_WIDE_STAGES:
        if (value != 2 && value != 3) return fail(ctx, BPMAX_EINVAL, "tile-product stages must be 2 or 3");
        ctx->wide_stages = (int)value;
        break;
    case BPMAX_TUNE_R0_VARIANT:
        if (value != 0 && value != 1) return fail(ctx, BPMAX_EINVAL, "product shape variant must be 0 or 1");
        ctx->r0_variant = (int)value;
        break;
    case BPMAX_TUNE_CLASS_SHARE:
        ctx->class_share = value != 0;
        break;
    case BPMAX_TUNE_PERSISTENT:
        if (value < 0 || value > 2) return fail(ctx, BPMAX_EINVAL, "persistent mode must be 0, 1 or 2");
        ctx->persist = (int)value;
        break;
    default: return fail(ctx, BPMAX_EINVAL, "unknown tuning key %d", key);
    }
    return BPMAX_OK;
}

int bpmax_gpu_get_tuning(const bpmax_ctx *ctx, int key, long *value)
{
    if (!ctx || !value) return BPMAX_EINVAL;
    switch (key) {
    case BPMAX_TUNE_R0_PAIRS_PER_JOB: *value = ctx->r0_pairs_per_job; break;
    case BPMAX_TUNE_R0_MERGE_ITEMS: *value = ctx->r0_merge_items; break;
    case BPMAX_TUNE_CLASS_STREAMS: *value = ctx->class_streams; break;
    case BPMAX_TUNE_WAIT_LIMIT_US: *value = (long)(ctx->wait_ns / 1000ULL); break;
    case BPMAX_TUNE_INJECT_WAIT_TIMEOUT: *value = ctx->inject_wait_timeout ? 1 : 0; break;
    case BPMAX_TUNE_WIDE_STAGES: *value = ctx->wide_stages; break;
    case BPMAX_TUNE_R0_VARIANT: *value = ctx->r0_variant; break;
    case BPMAX_TUNE_CLASS_SHARE: *value = ctx->class_share; break;
    case BPMAX_TUNE_PERSISTENT: *value = ctx->persist; break;
    default: return BPMAX_EINVAL;
    }
    return BPMAX_OK;
}

int bpmax_gpu_autotune(bpmax_ctx *ctx, int num_pairs, const int *const *seq1s, const long *Ms, const int *const *seq2s,
                       const long *Ns, int trials, long *best, float *best_ms)
{
    if (!ctx) return BPMAX_EINVAL;
    if (num_pairs < 1 || !Ms || !Ns) return fail(ctx, BPMAX_EINVAL, "empty batch");
    std::vector<int> vm(num_pairs), vn(num_pairs);
    for (int p = 0; p < num_pairs; ++p) {
        vm[p] = (int)Ms[p];
        vn[p] = (int)Ns[p];
    }
    const std::vector<int> key = shape_key(vm, vn);
    ctx->tuned.erase(key);
    const Tuned saved{ctx->r0_pairs_per_job, ctx->r0_merge_items, ctx->class_streams, ctx->r0_variant,
                      ctx->wide_stages,      ctx->class_share,    ctx->persist};
    std::set<int> classes;
    bool small = false, tiled = false;
    for (int n : vn) {
        const int np = padded_width(n);
        classes.insert(np);
        small = small || np <= MAX_SMALL_NP;
        tiled = tiled || is_tiled(np);
    }
    float best_t = -1.f;
    Tuned best_cfg = saved;
    int st = BPMAX_OK;
    auto try_cfg = [&](const Tuned &c) {
        ctx->r0_pairs_per_job = c[0];
        ctx->r0_merge_items = c[1];
        ctx->class_streams = c[2];
        ctx->r0_variant = c[3];
        ctx->wide_stages = c[4];
        ctx->class_share = c[5];
        ctx->persist = c[6];
        float t = -1.f;
        for (int r = 0; r < 1 + std::max(1, trials) && st == BPMAX_OK; ++r) {  // first run captures the graph
            st = fill_pairs(ctx, num_pairs, seq1s, Ms, seq2s, Ns);
            if (st == BPMAX_OK && r > 0 && (t < 0 || ctx->last_ms < t)) t = ctx->last_ms;
        }
        if (st == BPMAX_OK && (best_t < 0 || t < best_t)) {
            best_t = t;
            best_cfg = c;
        }
    };
    // the schedule knobs with the default kernel shapes, then the kernel shapes with the best schedule
    const int jobs_cand[] = {8, 32, 1 << 20}, merge_cand[] = {1, 4}, streams_cand[] = {1, 0};
    for (int sc : streams_cand) {
        if (sc == 0 && classes.size() < 2) continue;  // one class: the stream setting changes nothing
        for (int jc : jobs_cand)
            for (int mc : merge_cand)
                if (st == BPMAX_OK) try_cfg(Tuned{jc, mc, sc, 0, 2, 0, 0});
    }
    if (classes.size() > 1 && best_cfg[2] == 1 && st == BPMAX_OK)
        try_cfg(Tuned{best_cfg[0], best_cfg[1], 1, 0, 2, 1, 0});
    const Tuned sched = best_cfg;
    if (small && st == BPMAX_OK) try_cfg(Tuned{sched[0], sched[1], sched[2], 1, sched[4], sched[5], 0});
    if (tiled && st == BPMAX_OK) try_cfg(Tuned{sched[0], sched[1], sched[2], best_cfg[3], 3, sched[5], 0});
    // the persistent fill, merge cost as found; several width classes one after another (side by side,
    // mode 1, they do not stay on their SM shares and measured 4.5x slower on the 512-pair batch)
    if (!tiled && st == BPMAX_OK)
        for (int jc : jobs_cand)
            if (st == BPMAX_OK) try_cfg(Tuned{jc, sched[1], sched[2], 0, sched[4], 0, classes.size() > 1 ? 2 : 1});
    ctx->r0_pairs_per_job = saved[0];
    ctx->r0_merge_items = saved[1];
    ctx->class_streams = saved[2];
    ctx->r0_variant = saved[3];
    ctx->wide_stages = saved[4];
    ctx->class_share = saved[5];
    ctx->persist = saved[6];
    if (st != BPMAX_OK) return st;
    ctx->tuned[key] = best_cfg;
    if (best)
        for (int k = 0; k < 7; ++k) best[k] = best_cfg[k];
    if (best_ms) *best_ms = best_t;
    return BPMAX_OK;
}

int bpmax_gpu_read_cells(bpmax_ctx *ctx, int pair, long i1_lo, long i1_hi, long j1_lo, long j1_hi, float *out)
{
    if (!ctx) return BPMAX_EINVAL;
    if (!ctx->plan_valid) return fail(ctx, BPMAX_EINVAL, "no fill has run on this context");
    const Plan &P = ctx->plan;
    if (pair < 0 || pair >= (int)P.pairs.size()) return fail(ctx, BPMAX_EINVAL, "pair %d out of range", pair);
    const PairDesc &pd = P.pairs[pair];
    if (!out || i1_lo < 0 || j1_lo < 0 || i1_lo >= i1_hi || j1_lo >= j1_hi || i1_hi > pd.M || j1_hi > pd.M)
        return fail(ctx, BPMAX_EINVAL, "outer cell window [%ld,%ld) x [%ld,%ld) outside 0..%d", i1_lo, i1_hi, j1_lo,
                    j1_hi, pd.M);
    CK(cudaSetDevice(ctx->device));
    const long long n_out = (long long)(i1_hi - i1_lo) * (j1_hi - j1_lo) * pd.N * pd.N;
    int st;
    if ((st = ensure(ctx, ctx->conv, n_out * sizeof(float))) != BPMAX_OK) return st;
    read_cells_kernel<<<4 * ctx->sms, 256, 0, ctx->stream>>>((const PairDesc *)ctx->pairs.p + pair, (const float *)ctx->F.p,
                                                             (int)i1_lo, (int)j1_lo, (int)(j1_hi - j1_lo), n_out,
                                                             (float *)ctx->conv.p);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, ctx->conv.p, n_out * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return BPMAX_OK;
}

int bpmax_gpu_last_timing(const bpmax_ctx *ctx, float *fill_ms, long *launches)
{
    if (!ctx) return BPMAX_EINVAL;
    if (fill_ms) *fill_ms = ctx->last_ms;
    if (launches) *launches = ctx->last_launches;
    return BPMAX_OK;
}

}  // extern "C"

// =========================================================================================
// Allocation-free score entry point (bpmax_gpu_score_noalloc).
//
// Some callers cannot allocate device memory: code that runs inside another framework's
// memory pool or under a fixed device-memory budget (where a raw cudaMalloc is forbidden or
// would exceed the budget), and latency-sensitive callers that must not risk the implicit
// device synchronisation cudaMalloc/cudaFree can cause. For them the fill's scratch (the F and
// FT tables, S1/S2, the sequences and the job lists) lives in one fixed file-scope device array
// instead of the context's arenas. Every GPU that loads this library holds that array until
// the process exits.
// =========================================================================================
namespace {

constexpr size_t NOALLOC_FLOATS = (size_t)16 << 20;  // 64 MiB of fp32 scratch
constexpr unsigned long long NOALLOC_WAIT_NS = 4000000000ULL;  // time limit of one bounded wait

static __device__ __align__(256) float g_noalloc_scratch[NOALLOC_FLOATS];

struct NoallocDevice {
    float *ptr = nullptr;  // device address of g_noalloc_scratch on this device
    int sms = 0;
    int occ[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};  // resident product CTAs per SM, per width class
};
std::mutex g_noalloc_mu;
constexpr int NOALLOC_MAX_DEVICES = 64;
NoallocDevice g_noalloc_dev[NOALLOC_MAX_DEVICES];

// sequences (int32, seq1 then seq2) -> base codes (seq1, then seq2 reversed); cell job list
__global__ void noalloc_prep_kernel(const int *__restrict__ seqs, int M, int N, uint8_t *__restrict__ bases,
                                    CellJob *__restrict__ cells)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < M + N; i += gridDim.x * blockDim.x) {
        bases[i] = (uint8_t)(i < M ? seqs[i] : seqs[M + (N - 1 - (i - M))]);
        if (i < M) cells[i] = CellJob{0, i};
    }
}

// product jobs of diagonal d: pair chunk c of q offset pairs for every cell (i1, i1+d), ordered by
// chunk then cell, as the context path orders them
__global__ void noalloc_r0_jobs_kernel(R0Job *__restrict__ jobs, int cells, int d, int q, int njobs)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= njobs) return;
    const int P2 = (d + 1) / 2, c = t / cells, i1 = t % cells;
    jobs[t] = R0Job{0, i1, c * q, min(c * q + q, P2)};
}

template <int NB>
int noalloc_set_attr(int *occ)
{
    if (cudaFuncSetAttribute(r0_kernel<NB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)R0Cfg<NB>::SMEM) !=
        cudaSuccess)
        return BPMAX_ECUDA;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[NB], r0_kernel<NB>, R0Cfg<NB>::THREADS, R0Cfg<NB>::SMEM) !=
        cudaSuccess)
        return BPMAX_ECUDA;
    return cudaFuncSetAttribute(finalize_small_kernel<8 * NB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)FinShape<8 * NB>::SMEM) == cudaSuccess ? BPMAX_OK : BPMAX_ECUDA;
}

// Once per device, with that device current: the device address of the scratch array (a host
// reference to g_noalloc_scratch is only a host-side stand-in) and the kernels' attributes.
int noalloc_setup(int dev, NoallocDevice *out)
{
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    NoallocDevice &nd = g_noalloc_dev[dev];
    if (!nd.ptr) {
        float *p = nullptr;
        if (cudaGetSymbolAddress((void **)&p, g_noalloc_scratch) != cudaSuccess || !p) {
            cudaGetLastError();
            return BPMAX_ECUDA;
        }
        int sms = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return BPMAX_ECUDA;
        int st = noalloc_set_attr<1>(nd.occ);
        if (!st) st = noalloc_set_attr<2>(nd.occ);
        if (!st) st = noalloc_set_attr<3>(nd.occ);
        if (!st) st = noalloc_set_attr<4>(nd.occ);
        if (!st) st = noalloc_set_attr<5>(nd.occ);
        if (!st) st = noalloc_set_attr<6>(nd.occ);
        if (!st) st = noalloc_set_attr<7>(nd.occ);
        if (!st) st = noalloc_set_attr<8>(nd.occ);
        if (st) return st;
        nd.sms = sms;
        nd.ptr = p;
    }
    *out = nd;
    return BPMAX_OK;
}

template <int NB>
void noalloc_launch_diag(cudaStream_t s, const NoallocDevice &nd, int d, int n_r0, int n_cells, const R0Job *rj,
                         const CellJob *cj, const PairDesc *pd, float *F, float *S, const uint8_t *bases, const Weights &W,
                         int *err)
{
    if (d > 0)
        r0_kernel<NB><<<std::min(n_r0, std::max(1, nd.occ[NB]) * nd.sms), R0Cfg<NB>::THREADS, R0Cfg<NB>::SMEM, s>>>(
            rj, n_r0, pd, F, d, WaitCtl{err, NOALLOC_WAIT_NS, 0});
    const int n_s1 = n_cells - 1;  // S1 cells of diagonal d+1: the first n_cells-1 entries of cj
    using Sh = FinShape<8 * NB>;
    finalize_small_kernel<8 * NB><<<n_cells + (n_s1 + Sh::WARPS - 1) / Sh::WARPS, Sh::THREADS, Sh::SMEM, s>>>(
        cj, n_cells, cj, n_s1, pd, F, S, bases, W, d, RefOut{nullptr, 0, 0});
}

}  // namespace

extern "C" int bpmax_gpu_score_noalloc(const int *seq1, long M, const int *seq2, long N, const float *weights12,
                                       float *score, void *stream)
{
    if (!seq1 || !seq2 || !weights12 || !score || M < 1 || N < 1 || M > 65535 || N > MAX_SMALL_NP)
        return BPMAX_EINVAL;
    for (long i = 0; i < M; ++i)
        if (seq1[i] < 0 || seq1[i] > 4) return BPMAX_EINVAL;
    for (long i = 0; i < N; ++i)
        if (seq2[i] < 0 || seq2[i] > 4) return BPMAX_EINVAL;
    if (!weights_ok(weights12)) return BPMAX_EINVAL;
    // an error left pending by the caller's own earlier work is not this call's to report or clear
    if (cudaPeekAtLastError() != cudaSuccess) return BPMAX_ECUDA;
    const int Np = std::max(8, (int)(N + 7) / 8 * 8);
    const int nb = Np / 8;
    // scratch layout (floats), every region 256-byte aligned
    const long long nF = (long long)M * (M + 1) / 2 * cell_floats(Np);
    const long long off_S = align64(nF);
    const long long S2_rel = align64((long long)M * M);
    const long long S2m_rel = S2_rel + align64((long long)Np * Np), S2t_rel = S2m_rel + align64((long long)Np * Np);
    const long long off_seq = off_S + S2t_rel + align64((long long)Np * Np);
    const long long off_bases = off_seq + align64(M + N);
    const long long off_pd = off_bases + align64((M + N + 3) / 4);
    const long long off_score = off_pd + align64((long long)(sizeof(PairDesc) + 3) / 4);  // score, error flag
    const long long off_cj = off_score + 64;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEVICES) {
        cudaGetLastError();
        return BPMAX_ENODEV;
    }
    NoallocDevice nd;
    int st = noalloc_setup(dev, &nd);
    if (st) return st;
    const long long resident = (long long)std::max(1, nd.occ[nb]) * nd.sms;
    const int qmin = std::max(1, (R0_TAB_ITEMS[nb] + 1) / 2);
    // jobs per diagonal <= M * ceil(P2 / qmin) <= M * ((M + 1) / 2)
    const long long off_rj = off_cj + align64(2LL * M);
    const long long max_jobs = (long long)M * (((M + 1) / 2 + qmin - 1) / qmin);
    const long long total = off_rj + 4LL * max_jobs;
    if ((size_t)total > NOALLOC_FLOATS) return BPMAX_EINVAL;  // pair too large for the fixed scratch

    cudaStream_t s = (cudaStream_t)stream;
    float *base = nd.ptr;
    float *F = base, *S = base + off_S;
    int *seqs = reinterpret_cast<int *>(base + off_seq);
    uint8_t *bases = reinterpret_cast<uint8_t *>(base + off_bases);
    PairDesc *pdp = reinterpret_cast<PairDesc *>(base + off_pd);
    float *dscore = base + off_score;
    int *derr = reinterpret_cast<int *>(base + off_score + 1);
    CellJob *cj = reinterpret_cast<CellJob *>(base + off_cj);
    R0Job *rj = reinterpret_cast<R0Job *>(base + off_rj);
    PairDesc pd{};
    pd.M = (int)M;
    pd.N = (int)N;
    pd.Np = Np;
    pd.F_off = 0;
    pd.S1_off = 0;
    pd.S2_off = S2_rel;
    pd.S2m_off = S2m_rel;
    pd.S2t_off = S2t_rel;
    pd.seq1_off = 0;
    pd.seq2_off = (int)M;
    Weights W;
    memcpy(W.w, weights12, sizeof W.w);

    auto ok = [](cudaError_t e) { return e == cudaSuccess; };
    // pageable host sources: the copies are staged before cudaMemcpyAsync returns
    if (!ok(cudaMemcpyAsync(seqs, seq1, sizeof(int) * M, cudaMemcpyHostToDevice, s)) ||
        !ok(cudaMemcpyAsync(seqs + M, seq2, sizeof(int) * N, cudaMemcpyHostToDevice, s)) ||
        !ok(cudaMemcpyAsync(pdp, &pd, sizeof pd, cudaMemcpyHostToDevice, s)) ||
        !ok(cudaMemsetAsync(F, 0, sizeof(float) * nF, s)) ||        // F starts at +0 on every call
        !ok(cudaMemsetAsync(S, 0, sizeof(float) * S2_rel, s)) ||    // and S1 at 0
        !ok(cudaMemsetAsync(derr, 0, sizeof(int), s))) {
        cudaGetLastError();
        return BPMAX_ECUDA;
    }
    noalloc_prep_kernel<<<8, 256, 0, s>>>(seqs, (int)M, (int)N, bases, cj);
    single_strand_kernel<<<1, 512, 0, s>>>(pdp, bases, S, W);
    s2_aux_kernel<<<1, 256, 0, s>>>(pdp, S);
    for (int d = 0; d < (int)M; ++d) {
        const int cells = (int)M - d;
        int n_r0 = 0;
        if (d > 0) {
            const long long P2 = (d + 1) / 2;
            const long long q = r0_pairs_per_job(cells, P2, resident, qmin, 1 << 20, 2);
            n_r0 = (int)(cells * ((P2 + q - 1) / q));
            noalloc_r0_jobs_kernel<<<(n_r0 + 255) / 256, 256, 0, s>>>(rj, cells, d, (int)q, n_r0);
        }
        switch (nb) {
        case 1: noalloc_launch_diag<1>(s, nd, d, n_r0, cells, rj, cj, pdp, F, S, bases, W, derr); break;
        case 2: noalloc_launch_diag<2>(s, nd, d, n_r0, cells, rj, cj, pdp, F, S, bases, W, derr); break;
        case 3: noalloc_launch_diag<3>(s, nd, d, n_r0, cells, rj, cj, pdp, F, S, bases, W, derr); break;
        case 4: noalloc_launch_diag<4>(s, nd, d, n_r0, cells, rj, cj, pdp, F, S, bases, W, derr); break;
        case 5: noalloc_launch_diag<5>(s, nd, d, n_r0, cells, rj, cj, pdp, F, S, bases, W, derr); break;
        case 6: noalloc_launch_diag<6>(s, nd, d, n_r0, cells, rj, cj, pdp, F, S, bases, W, derr); break;
        case 7: noalloc_launch_diag<7>(s, nd, d, n_r0, cells, rj, cj, pdp, F, S, bases, W, derr); break;
        default: noalloc_launch_diag<8>(s, nd, d, n_r0, cells, rj, cj, pdp, F, S, bases, W, derr); break;
        }
    }
    gather_scores_kernel<<<1, 32, 0, s>>>(pdp, F, 1, dscore);
    float out[2] = {0.f, 0.f};  // score, error flag bits
    if (!ok(cudaGetLastError()) || !ok(cudaMemcpyAsync(out, dscore, 2 * sizeof(float), cudaMemcpyDeviceToHost, s)) ||
        !ok(cudaStreamSynchronize(s))) {
        cudaGetLastError();
        return BPMAX_ECUDA;
    }
    int errbits = 0;
    memcpy(&errbits, &out[1], sizeof errbits);
    if (errbits != 0) return BPMAX_ETIMEOUT;
    *score = out[0];
    return BPMAX_OK;
}
