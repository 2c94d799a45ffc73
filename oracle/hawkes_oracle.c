/*
 * ORACLE -- TEST INFRASTRUCTURE ONLY.  Nothing in the product links, loads or
 * calls this file; only tests/, the smoke check and bench.py's CPU-baseline leg
 * do, and there only as the checker.
 *
 * A plain-C restatement of the hpHawkes spatio-temporal Hawkes log-likelihood
 * (the reference's CPU engine, src/NewHawkes.hpp) together with its analytic
 * parameter gradient, which the reference does not expose.  Parity pins:
 *   - loglik and probs are checked against the reference engine itself,
 *     compiled from its sources into oracle/_ref (tests/test_oracle.py) and
 *     against golden fixtures generated from it (tests/golden/);
 *   - the gradient is checked against central finite differences of the
 *     reference engine's loglik.
 *
 * Model (parameters are precisions; order follows NewHawkes::setParameters,
 * src/NewHawkes.hpp:331-339: sigma, a=tauX, b=tauT, omega, theta, mu0):
 *   phi(v)  = exp(-v^2/2)/sqrt(2 pi)                    (src/NewHawkes.hpp:108-111)
 *   B_ij    = mu0 a^D b phi(a d_ij) phi(b dt_ij), all j  (src/NewHawkes.hpp:538-539)
 *   S_ij    = theta omega sigma^D phi(sigma d_ij) exp(-omega dt_ij), dt_ij > 0
 *                                                        (src/NewHawkes.hpp:540-541)
 *   lam_i   = sum_j B_ij + S_ij                          (src/NewHawkes.hpp:533-546)
 *   ll_i    = log lam_i + theta (exp(-omega (T - t_i)) - 1)
 *             - mu0 (Phi(b (T - t_i)) - Phi(-b t_i))      (src/NewHawkes.hpp:652-655)
 *   logL    = sum_i ll_i + N (D - 1) log(1/sqrt(2 pi))    (src/NewHawkes.hpp:659)
 *   P_i     = sum_j S_ij / lam_i                         (src/NewHawkes.hpp:685)
 * with d_ij the Euclidean distance (src/Distance.hpp:72-83), dt_ij = t_i - t_j,
 * T = t_{N-1} (src/NewHawkes.hpp:653) and Phi(v) = exp(log(0.5 erfc(-v/sqrt2)))
 * (src/CDF.h:584-592).  An independent statement of the same model is the
 * reference's naive R code, R/log_lik_and_grad.R:2-93.
 *
 * Gradient, derived here from the model above (the reference's own gradient
 * code at src/NewHawkes.hpp:341-402, :592-634 is dead and does not match the
 * live model).  With Sb = sum_j B_ij, Sbd = sum_j B_ij d^2, Sbt = sum_j B_ij dt^2,
 * Ss = sum_j S_ij, Ssd = sum_j S_ij d^2, Sst = sum_j S_ij dt, D_i = T - t_i:
 *   dlogL/dsigma = sum_i (D/sigma Ss - sigma Ssd)/lam_i
 *   dlogL/da     = sum_i (D/a Sb - a Sbd)/lam_i
 *   dlogL/db     = sum_i (Sb/b - b Sbt)/lam_i - mu0 (phi(b D_i) D_i + phi(b t_i) t_i)
 *   dlogL/domega = sum_i (Ss/omega - Sst)/lam_i - theta D_i exp(-omega D_i)
 *   dlogL/dtheta = sum_i (Ss/theta)/lam_i + exp(-omega D_i) - 1
 *   dlogL/dmu0   = sum_i (Sb/mu0)/lam_i - (Phi(b D_i) - Phi(-b t_i))
 *
 * Pair sums are accumulated in long double (x87 80-bit) over j and the final
 * sum over i in long double in index order, so results do not depend on the
 * thread count.  Each pair term itself is an IEEE double computed with libm.
 */
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_INV_SQRT_2PI 0.398942280401432677939946059934
#define ORACLE_SQRT1_2 0.707106781186547524401

static double oracle_phi(double v) { return ORACLE_INV_SQRT_2PI * exp(-0.5 * v * v); }
static double oracle_Phi(double v) { return exp(log(0.5 * erfc(-v * ORACLE_SQRT1_2))); }

typedef struct {
    int D, N;
    const double* loc;
    const double* t;
    double sigma, a, b, omega, theta, mu0;
    int i0, i1;
    /* per-event outputs (length N, or 6N for grads) */
    double* ll;        /* ll_i without the constant */
    double* g;         /* 6 per event */
    double* gabs;      /* 6 per event: |pair part| + |compensator part| */
    double* gterm;     /* 6 per event: sum of |every additive term|; may be null */
    double* probs;     /* may be null */
    double* lam;       /* may be null */
    double* sums;      /* may be null: 6 per event, the unit pair sums */
} oracle_job;

static void* oracle_worker(void* arg) {
    oracle_job* J = (oracle_job*)arg;
    const int D = J->D, N = J->N;
    const double sigma = J->sigma, a = J->a, b = J->b, omega = J->omega, theta = J->theta,
                 mu0 = J->mu0;
    /* prefactors without the leading theta / mu0 so that theta = 0 or mu0 = 0 stay finite */
    const double bgScale = pow(a, D) * b;          /* B_ij = mu0 bgScale phi(a d) phi(b dt) */
    const double seScale = omega * pow(sigma, D);  /* S_ij = theta seScale phi(s d) e^{-w dt} */
    const double T = J->t[N - 1];
    for (int i = J->i0; i < J->i1; ++i) {
        long double sb = 0, sbd = 0, sbt = 0, ss = 0, ssd = 0, sst = 0;
        const double ti = J->t[i];
        const double* xi = J->loc + (size_t)i * D;
        for (int j = 0; j < N; ++j) {
            const double* xj = J->loc + (size_t)j * D;
            double d2 = 0.0;
            for (int k = 0; k < D; ++k) {
                const double diff = xi[k] - xj[k];
                d2 += diff * diff;
            }
            const double dist = sqrt(d2);
            const double dt = ti - J->t[j];
            const double bu = oracle_phi(a * dist) * oracle_phi(b * dt);
            sb += bu;
            sbd += (long double)bu * d2;
            sbt += (long double)bu * dt * dt;
            if (dt > 0.0) {
                const double su = oracle_phi(sigma * dist) * exp(-omega * dt);
                ss += su;
                ssd += (long double)su * d2;
                sst += (long double)su * dt;
            }
        }
        const long double SB = mu0 * bgScale * sb, SS = theta * seScale * ss;
        const long double lam = SB + SS;
        const double Di = T - ti;
        const double eW = exp(-omega * Di);
        const double cdfTerm = oracle_Phi(b * Di) - oracle_Phi(-b * ti);
        J->ll[i] = (double)(logl(lam) + (long double)theta * (eW - 1.0) - (long double)mu0 * cdfTerm);

        const long double SBd = mu0 * bgScale * sbd, SBt = mu0 * bgScale * sbt;
        const long double SSd = theta * seScale * ssd, SSt = theta * seScale * sst;
        long double pair[6], comp[6];
        pair[0] = ((long double)D / sigma * SS - sigma * SSd) / lam;
        comp[0] = 0;
        pair[1] = ((long double)D / a * SB - a * SBd) / lam;
        comp[1] = 0;
        pair[2] = (SB / b - b * SBt) / lam;
        comp[2] = -(long double)mu0 * (oracle_phi(b * Di) * Di + oracle_phi(b * ti) * ti);
        pair[3] = (SS / omega - SSt) / lam;
        comp[3] = -(long double)theta * Di * eW;
        pair[4] = (seScale * ss) / lam;
        comp[4] = eW - 1.0;
        pair[5] = (bgScale * sb) / lam;
        comp[5] = -cdfTerm;
        /* term-level scale: every additive term of the per-event contribution
         * in absolute value (the condition scale of the sum) */
        long double term[6];
        term[0] = (fabsl((long double)D / sigma * SS) + fabsl(sigma * SSd)) / lam;
        term[1] = (fabsl((long double)D / a * SB) + fabsl(a * SBd)) / lam;
        term[2] = (fabsl(SB / b) + fabsl(b * SBt)) / lam +
                  fabsl((long double)mu0 * oracle_phi(b * Di) * Di) +
                  fabsl((long double)mu0 * oracle_phi(b * ti) * ti);
        term[3] = (fabsl(SS / omega) + fabsl(SSt)) / lam + fabsl(comp[3]);
        term[4] = fabsl(pair[4]) + fabsl((long double)eW) + 1.0L;
        term[5] = fabsl(pair[5]) + fabsl((long double)oracle_Phi(b * Di)) +
                  fabsl((long double)oracle_Phi(-b * ti));
        for (int k = 0; k < 6; ++k) {
            J->g[(size_t)6 * i + k] = (double)(pair[k] + comp[k]);
            J->gabs[(size_t)6 * i + k] = (double)(fabsl(pair[k]) + fabsl(comp[k]));
            if (J->gterm) J->gterm[(size_t)6 * i + k] = (double)term[k];
        }
        if (J->probs) J->probs[i] = (double)(SS / lam);
        if (J->lam) J->lam[i] = (double)lam;
        if (J->sums) {
            double* s = J->sums + (size_t)6 * i;
            s[0] = (double)sb; s[1] = (double)sbd; s[2] = (double)sbt;
            s[3] = (double)ss; s[4] = (double)ssd; s[5] = (double)sst;
        }
    }
    return NULL;
}

/*
 * Evaluate the log-likelihood, its gradient (6, reference parameter order),
 * two absolute scales of the gradient (6 each): gradAbs = sum_i of
 * |per-event contribution| and gradTerm = sum_i of the absolute values of every
 * additive term of the per-event contribution (the condition scale of the
 * sum; optional), the self-excitation probabilities (N, optional) and the rates
 * lam_i (N, optional) for one parameter vector.  loc is row-major N x D (src/NewHawkes.hpp:244-276),
 * t has N entries.  Returns 0 on success, -1 on bad arguments.
 */
int hawkes_oracle_eval(int D, int N, const double* loc, const double* t, const double* params,
                       int nthreads, double* loglik, double* grad, double* gradAbs,
                       double* gradTerm, double* probs, double* lam) {
    if (D < 1 || N < 1 || !loc || !t || !params) return -1;
    if (nthreads < 1) nthreads = 1;
    if (nthreads > N) nthreads = N;
    double* ll = (double*)malloc(sizeof(double) * (size_t)N);
    double* g = (double*)malloc(sizeof(double) * (size_t)N * 6);
    double* ga = (double*)malloc(sizeof(double) * (size_t)N * 6);
    double* gm = (double*)malloc(sizeof(double) * (size_t)N * 6);
    oracle_job* jobs = (oracle_job*)calloc((size_t)nthreads, sizeof(oracle_job));
    pthread_t* th = (pthread_t*)calloc((size_t)nthreads, sizeof(pthread_t));
    if (!ll || !g || !ga || !gm || !jobs || !th) {
        free(ll); free(g); free(ga); free(gm); free(jobs); free(th);
        return -1;
    }
    const int chunk = (N + nthreads - 1) / nthreads;
    for (int k = 0; k < nthreads; ++k) {
        oracle_job* J = &jobs[k];
        J->D = D; J->N = N; J->loc = loc; J->t = t;
        J->sigma = params[0]; J->a = params[1]; J->b = params[2];
        J->omega = params[3]; J->theta = params[4]; J->mu0 = params[5];
        J->i0 = k * chunk;
        J->i1 = (k + 1) * chunk < N ? (k + 1) * chunk : N;
        if (J->i0 > N) J->i0 = N;
        J->ll = ll; J->g = g; J->gabs = ga; J->gterm = gm; J->probs = probs; J->lam = lam;
        J->sums = NULL;
    }
    for (int k = 1; k < nthreads; ++k) pthread_create(&th[k], NULL, oracle_worker, &jobs[k]);
    oracle_worker(&jobs[0]);
    for (int k = 1; k < nthreads; ++k) pthread_join(th[k], NULL);

    long double total = 0, gt[6] = {0, 0, 0, 0, 0, 0}, gat[6] = {0, 0, 0, 0, 0, 0};
    long double gmt[6] = {0, 0, 0, 0, 0, 0};
    for (int i = 0; i < N; ++i) {
        total += ll[i];
        for (int k = 0; k < 6; ++k) {
            gt[k] += g[(size_t)6 * i + k];
            gat[k] += ga[(size_t)6 * i + k];
            gmt[k] += gm[(size_t)6 * i + k];
        }
    }
    total += (long double)N * (D - 1) * logl(ORACLE_INV_SQRT_2PI);
    if (loglik) *loglik = (double)total;
    for (int k = 0; k < 6; ++k) {
        if (grad) grad[k] = (double)gt[k];
        if (gradAbs) gradAbs[k] = (double)gat[k];
        if (gradTerm) gradTerm[k] = (double)gmt[k];
    }
    free(ll); free(g); free(ga); free(gm); free(jobs); free(th);
    return 0;
}

/*
 * The six unit pair sums per event (no prefactors):
 *   sum_j phi(a d)phi(b dt) [1, d^2, dt^2]  and  sum_{dt>0} phi(s d)e^{-w dt} [1, d^2, dt],
 * written to sums (6 per event).  Used to check the device partial sums.
 */
int hawkes_oracle_pair_sums(int D, int N, const double* loc, const double* t, const double* params,
                            int nthreads, double* sums) {
    if (D < 1 || N < 1 || !loc || !t || !params || !sums) return -1;
    if (nthreads < 1) nthreads = 1;
    if (nthreads > N) nthreads = N;
    double* ll = (double*)malloc(sizeof(double) * (size_t)N);
    double* g = (double*)malloc(sizeof(double) * (size_t)N * 6);
    double* ga = (double*)malloc(sizeof(double) * (size_t)N * 6);
    oracle_job* jobs = (oracle_job*)calloc((size_t)nthreads, sizeof(oracle_job));
    pthread_t* th = (pthread_t*)calloc((size_t)nthreads, sizeof(pthread_t));
    if (!ll || !g || !ga || !jobs || !th) {
        free(ll); free(g); free(ga); free(jobs); free(th);
        return -1;
    }
    const int chunk = (N + nthreads - 1) / nthreads;
    for (int k = 0; k < nthreads; ++k) {
        oracle_job* J = &jobs[k];
        J->D = D; J->N = N; J->loc = loc; J->t = t;
        J->sigma = params[0]; J->a = params[1]; J->b = params[2];
        J->omega = params[3]; J->theta = params[4]; J->mu0 = params[5];
        J->i0 = k * chunk;
        J->i1 = (k + 1) * chunk < N ? (k + 1) * chunk : N;
        if (J->i0 > N) J->i0 = N;
        J->ll = ll; J->g = g; J->gabs = ga; J->gterm = NULL; J->probs = NULL; J->lam = NULL;
        J->sums = sums;
    }
    for (int k = 1; k < nthreads; ++k) pthread_create(&th[k], NULL, oracle_worker, &jobs[k]);
    oracle_worker(&jobs[0]);
    for (int k = 1; k < nthreads; ++k) pthread_join(th[k], NULL);
    free(ll); free(g); free(ga); free(jobs); free(th);
    return 0;
}
