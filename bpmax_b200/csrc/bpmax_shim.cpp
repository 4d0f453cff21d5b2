// bpmax_shim.cpp -- the reference's fill entry point, served by the GPU engine.
//
//   void bpmax(long M, long N, long N_sec, long N_tile, long R, long MR, long NR, long P,
//              int* seq1, int* seq2, float****** FTable)
// has the signature (and C++ linkage) of TPDS/source/release/MPT_RT_V3/
// bpmax_complete_otf_ftable/src/bpmax.c:129, so the reference's CLI wrapper
// (V3/bpmax-wrapper.c:277) links against libbpmax_gpu.so in place of the CPU objects.
// Parameter checking, message and exit code follow V3/bpmax.c:131-134. MR, NR and P tune the
// CPU register tiles and thread count; the GPU ignores them. R is recomputed from N and N_tile
// (the wrapper leaves it uninitialised when N % N_tile == 0, V3/bpmax-wrapper.c:158-167).
// Weights are the reference's hard-coded ones unless bpmax_gpu_shim_set_weights() changed them.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/bpmax_gpu.h"

namespace {
std::mutex g_mu;
bpmax_ctx *g_ctx = nullptr;
float g_w[12] = {1.0f, 1.0f, 3.0f, 3.0f, 1.5f, 1.5f, 1.0f, 1.0f, 3.0f, 3.0f, 1.5f, 1.5f};

[[noreturn]] void die(const char *msg)
{
    printf("%s\n", msg);
    exit(-1);
}
}  // namespace

extern "C" int bpmax_gpu_shim_set_weights(const float *w12)
{
    if (!w12) return BPMAX_EINVAL;
    for (int t = 0; t < 12; ++t)
        if (!std::isfinite(w12[t]) || w12[t] < 0.0f || std::signbit(w12[t])) return BPMAX_EINVAL;
    std::lock_guard<std::mutex> lk(g_mu);
    memcpy(g_w, w12, sizeof g_w);
    return BPMAX_OK;
}

void bpmax(long M, long N, long N_sec, long N_tile, long R, long MR, long NR, long P, int *seq1, int *seq2,
           float ******FTable)
{
    (void)R;
    if (!((M >= 1 && N >= 8 && N_sec >= 2 && N_tile >= 4 && MR >= 1 && NR >= 1 && P >= 1 && 0 >= P - 128)))
        die("The value of parameters are not valid.");
    const long Rc = (N_tile - N % N_tile) % N_tile;
    if (N_sec != (N + N_tile - 1) / N_tile || !(N_tile >= Rc + 1)) die("The value of parameters are not valid.");
    std::lock_guard<std::mutex> lk(g_mu);
    int st;
    if (!g_ctx && (st = bpmax_gpu_create(0, &g_ctx)) != BPMAX_OK) {
        fprintf(stderr, "bpmax: %s\n", bpmax_gpu_status_string(st));
        exit(-1);
    }
    if ((st = bpmax_gpu_set_weights(g_ctx, g_w)) != BPMAX_OK) die(bpmax_gpu_last_error(g_ctx));
    // The wrapper's pointer tree sits over one linear buffer (V3/bpmax-wrapper.c:192); fill it
    // directly when that holds, otherwise through a contiguous copy and the tree.
    float *base = &FTable[0][0][0][0][0][0];
    const long T = N_tile, Ns = N_sec;
    float *last = &FTable[M - 1][M - 1][Ns - 1][Ns - 1][T][0];
    const long expect = ((((M - 1) * M + (M - 1)) * Ns + (Ns - 1)) * Ns + (Ns - 1)) * (T + 1) * T + T * T;
    if (last - base == expect) {
        st = bpmax_gpu_fill(g_ctx, seq1, M, seq2, N, N_tile, base, nullptr);
        if (st != BPMAX_OK) die(bpmax_gpu_last_error(g_ctx));
        return;
    }
    std::vector<float> lin((size_t)M * M * Ns * Ns * (T + 1) * T);
    st = bpmax_gpu_fill(g_ctx, seq1, M, seq2, N, N_tile, lin.data(), nullptr);
    if (st != BPMAX_OK) die(bpmax_gpu_last_error(g_ctx));
    for (long a = 0; a < M; ++a)
        for (long b = a; b < M; ++b)
            for (long c = 0; c < Ns; ++c)
                for (long d = c; d < Ns; ++d)
                    for (long e = 0; e <= T; ++e)
                        memcpy(FTable[a][b][c][d][e], &lin[((((a * M + b) * Ns + c) * Ns + d) * (T + 1) + e) * T],
                               sizeof(float) * T);
}
