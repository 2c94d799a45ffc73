/*
 * ORACLE / TEST INFRASTRUCTURE: a driver for hawkes_oracle.c built with
 * AddressSanitizer and UndefinedBehaviorSanitizer (tests/test_oracle_sanitized.py
 * compiles and runs it).  The oracle is the checker every parity test trusts,
 * so its memory and arithmetic safety is checked on the edge cases the tests
 * feed it: N = 1 and 2, sizes around the tiling blocks, D = 1..8, tied and
 * unsorted times, more threads than events, and rejected arguments.  Every
 * result must be finite and independent of the thread count.  Prints "ok"
 * and exits 0; any sanitizer report aborts with a non-zero status.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

int hawkes_oracle_eval(int D, int N, const double* loc, const double* t, const double* params,
                       int nthreads, double* loglik, double* grad, double* gradAbs,
                       double* gradTerm, double* probs, double* lam);
int hawkes_oracle_pair_sums(int D, int N, const double* loc, const double* t,
                            const double* params, int nthreads, double* sums);

static unsigned long long state = 88172645463325252ULL;
static double uniform(void) { /* xorshift64 */
    state ^= state << 13;
    state ^= state >> 7;
    state ^= state << 17;
    return (double)(state >> 11) * (1.0 / 9007199254740992.0);
}

static int fail(const char* what, int D, int N) {
    fprintf(stderr, "FAILED: %s (D=%d, N=%d)\n", what, D, N);
    return 1;
}

static int check_case(int D, int N, int ties, int unsorted) {
    double* loc = malloc(sizeof(double) * (size_t)N * D);
    double* t = malloc(sizeof(double) * (size_t)N);
    double* probs[2] = {malloc(sizeof(double) * N), malloc(sizeof(double) * N)};
    double* lam = malloc(sizeof(double) * N);
    double* sums[2] = {malloc(sizeof(double) * 6 * N), malloc(sizeof(double) * 6 * N)};
    const double params[6] = {1.0, 1.0 / 1.6, 1.0 / 336.0, 1.0, 1.0, 1.0};
    int bad = 0;
    for (int i = 0; i < N * D; ++i) loc[i] = 20.0 * uniform();
    for (int i = 0; i < N; ++i) t[i] = 8760.0 * (double)i / N;
    if (ties)
        for (int i = 0; i < N; ++i) t[i] = floor(t[i] / 500.0) * 500.0;
    if (unsorted)
        for (int i = 0; i + 1 < N; i += 2) {
            const double s = t[i];
            t[i] = t[i + 1];
            t[i + 1] = s;
        }
    double ll[2], g[2][6], ga[6], gm[6];
    const int threads[2] = {1, 5};
    for (int k = 0; k < 2; ++k) {
        if (hawkes_oracle_eval(D, N, loc, t, params, threads[k], &ll[k], g[k], ga, gm, probs[k],
                               lam) != 0)
            bad |= fail("eval returned an error", D, N);
        if (hawkes_oracle_pair_sums(D, N, loc, t, params, threads[k], sums[k]) != 0)
            bad |= fail("pair sums returned an error", D, N);
    }
    if (!isfinite(ll[0])) bad |= fail("non-finite log-likelihood", D, N);
    if (ll[0] != ll[1]) bad |= fail("log-likelihood depends on the thread count", D, N);
    for (int q = 0; q < 6; ++q)
        if (!isfinite(g[0][q]) || g[0][q] != g[1][q] || !isfinite(ga[q]) || !isfinite(gm[q]))
            bad |= fail("gradient not finite or thread-dependent", D, N);
    for (int i = 0; i < N; ++i)
        if (!(probs[0][i] >= 0.0 && probs[0][i] <= 1.0) || probs[0][i] != probs[1][i] ||
            !(lam[i] > 0.0))
            bad |= fail("probabilities or rates out of range", D, N);
    if (memcmp(sums[0], sums[1], sizeof(double) * 6 * N) != 0)
        bad |= fail("pair sums depend on the thread count", D, N);
    free(loc);
    free(t);
    free(probs[0]);
    free(probs[1]);
    free(lam);
    free(sums[0]);
    free(sums[1]);
    return bad;
}

int main(void) {
    int bad = 0;
    const int sizes[] = {1, 2, 3, 31, 32, 33, 127, 128, 129, 257};
    for (int D = 1; D <= 8; ++D)
        for (size_t s = 0; s < sizeof sizes / sizeof sizes[0]; ++s)
            bad |= check_case(D, sizes[s], s % 2, s % 3 == 0);
    /* rejected arguments return -1 without touching memory */
    const double p[6] = {1, 1, 1, 1, 1, 1}, x[2] = {0, 0}, t[1] = {0};
    double ll, sums[6];
    if (hawkes_oracle_eval(0, 1, x, t, p, 1, &ll, NULL, NULL, NULL, NULL, NULL) != -1 ||
        hawkes_oracle_eval(2, 0, x, t, p, 1, &ll, NULL, NULL, NULL, NULL, NULL) != -1 ||
        hawkes_oracle_eval(2, 1, NULL, t, p, 1, &ll, NULL, NULL, NULL, NULL, NULL) != -1 ||
        hawkes_oracle_pair_sums(2, 1, x, t, p, 1, NULL) != -1 ||
        hawkes_oracle_pair_sums(2, 1, x, NULL, p, 1, sums) != -1)
        bad |= fail("bad arguments not rejected", 0, 0);
    if (bad) return 1;
    printf("ok\n");
    return 0;
}
