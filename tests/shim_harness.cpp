// Drop-in check: a caller written like the reference's CLI wrapper (V3/bpmax-wrapper.c:175-197
// allocation, :277 call) links against libbpmax_gpu.so and calls the C++ bpmax() symbol.
// Usage: shim_harness M N N_tile out.bin [w1 .. w12]  (reads M then N base codes from stdin;
// with 12 weights, sets them through bpmax_gpu_shim_set_weights before the call)
#include <cstdio>
#include <cstdlib>
void bpmax(long, long, long, long, long, long, long, long, int *, int *, float ******);
extern "C" int bpmax_gpu_shim_set_weights(const float *w12);
int main(int argc, char **argv)
{
    if (argc < 5) return 2;
    if (argc >= 17) {
        float w[12];
        for (int t = 0; t < 12; ++t) w[t] = (float)atof(argv[5 + t]);
        if (bpmax_gpu_shim_set_weights(w) != 0) return 4;
    }
    long M = atol(argv[1]), N = atol(argv[2]), T = atol(argv[3]);
    long Ns = (N + T - 1) / T, R = (T - N % T) % T;
    int *s1 = (int *)malloc(sizeof(int) * M), *s2 = (int *)malloc(sizeof(int) * N);
    for (long i = 0; i < M; ++i) if (scanf("%d", &s1[i]) != 1) return 3;
    for (long i = 0; i < N; ++i) if (scanf("%d", &s2[i]) != 1) return 3;
    size_t n = (size_t)M * M * Ns * Ns * (T + 1) * T;
    float *lin = (float *)malloc(sizeof(float) * n);
    for (size_t i = 0; i < n; ++i) lin[i] = __builtin_nanf("");
    float ******F = (float ******)malloc(sizeof(float *****) * M);
    for (long a = 0; a < M; ++a) {
        F[a] = (float *****)malloc(sizeof(float ****) * M);
        for (long b = 0; b < M; ++b) {
            F[a][b] = (float ****)malloc(sizeof(float ***) * Ns);
            for (long c = 0; c < Ns; ++c) {
                F[a][b][c] = (float ***)malloc(sizeof(float **) * Ns);
                for (long d = 0; d < Ns; ++d) {
                    F[a][b][c][d] = (float **)malloc(sizeof(float *) * (T + 1));
                    for (long e = 0; e <= T; ++e) F[a][b][c][d][e] = &lin[((((a * M + b) * Ns + c) * Ns + d) * (T + 1) + e) * T];
                }
            }
        }
    }
    bpmax(M, N, Ns, T, R, 3, 8, 8, s1, s2, F);
    FILE *f = fopen(argv[4], "wb");
    fwrite(lin, sizeof(float), n, f);
    fclose(f);
    printf("F(0,%ld,0,%ld)=%10e\n", M - 1, N - 1, F[0][M - 1][(0 + R) / T][(N - 1 + R) / T][(0 + R) % T][(N - 1 + R) % T]);
    return 0;
}
