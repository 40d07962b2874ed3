/*
 * CPU oracle of the Clifford & Clifford Fock sampler (TEST INFRASTRUCTURE: only tests/, the smoke
 * check and bench.py's CPU-baseline arm may load it; the product path never does).
 *
 * A plain-C restatement of the reference's algorithm for the sampling path:
 *   photonic_engines/clifford/sampler.py:391-460          (the chain over steps, stream layout)
 *   photonic_engines/clifford/cofactors_triton.py:413-447 (multiplicity tables, halving rule)
 *   photonic_engines/clifford/cuda_cofactors.py:72-106    (reflected mixed-radix Gray odometer)
 *   photonic_engines/clifford/variants.py:70-114          (2020 cofactors, exact all-but-one)
 *   photonic_engines/clifford/cofactors_triton.py:287-308 (scale, amplitudes, 48-bit uniform, pick)
 *   triton/language/random.py (installed Triton, philox_impl / randint4x / uint_to_uniform_float):
 *       Philox4x32-10 (Salmon et al., SC'11) as the reference's draw kernel calls it through tl.rand.
 *
 * Built twice over one body (oracle_impl.h): REAL = double (suffix _f64) and REAL = long double
 * (suffix _ld, x87 80-bit, the extended-precision error reference).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <stdatomic.h>
#include <unistd.h>

#define ORACLE_MAXN 64

static double binom_tab[ORACLE_MAXN + 1][ORACLE_MAXN + 1];
static int binom_ready = 0;

static void init_binom(void) {
    if (binom_ready) return;
    for (int a = 0; a <= ORACLE_MAXN; ++a) {
        binom_tab[a][0] = 1.0;
        for (int b = 1; b <= a; ++b) binom_tab[a][b] = binom_tab[a][b - 1] * (double)(a - b + 1) / (double)b;
        for (int b = a + 1; b <= ORACLE_MAXN; ++b) binom_tab[a][b] = 0.0;
    }
    binom_ready = 1;
}

/* ------------------------------------------------------------------ Philox4x32-10, Triton flavour */

static uint32_t umulhi32(uint32_t a, uint32_t b) { return (uint32_t)(((uint64_t)a * (uint64_t)b) >> 32); }

/* randint4x(seed, offset)[0] of triton/language/random.py for a non-negative int32 offset and a
 * seed < 2^31: counter (offset, 0, 0, 0), key (seed_lo, seed_hi), 10 rounds.  */
uint32_t oracle_philox_randint(uint64_t seed, uint32_t offset) {
    uint32_t c0 = offset, c1 = 0, c2 = 0, c3 = 0;
    uint32_t k0 = (uint32_t)(seed & 0xffffffffu), k1 = (uint32_t)(seed >> 32);
    for (int r = 0; r < 10; ++r) {
        uint32_t o0 = c0, o2 = c2;
        c0 = umulhi32(0xCD9E8D57u, o2) ^ c1 ^ k0;
        c2 = umulhi32(0xD2511F53u, o0) ^ c3 ^ k1;
        c1 = 0xCD9E8D57u * o2;
        c3 = 0xD2511F53u * o0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c0;
}

/* uint_to_uniform_float for 32-bit draws: bitcast to int32, fold negatives (-x - 1), times the
 * float32 constant 4.6566127342e-10, all in float32 (int -> float rounds to nearest).  */
float oracle_triton_rand(uint64_t seed, uint32_t offset) {
    int32_t x = (int32_t)oracle_philox_randint(seed, offset);
    if (x < 0) x = -x - 1;
    volatile float xf = (float)x;
    volatile float r = xf * 4.6566127342e-10f;
    return r;
}

/* The draw kernel's 48-bit uniform of stream s at a step with seed `seed`:
 * u = (r0 + r1 * 2^-24) / (1 + 2^-24), r_i = tl.rand(seed, 2 s + i) (cofactors_triton.py:303-305).  */
double oracle_uniform(uint64_t seed, int64_t s) {
    volatile double r0 = (double)oracle_triton_rand(seed, (uint32_t)(2 * s));
    volatile double r1 = (double)oracle_triton_rand(seed, (uint32_t)(2 * s + 1));
    volatile double t = r1 * 5.9604644775390625e-08;
    volatile double num = r0 + t;
    return num / (1.0 + 5.9604644775390625e-08);
}

/* u [S][n]: the uniform of stream s (local index within its lockstep pass) at step k uses seeds[k].  */
void oracle_uniforms(const int64_t* seeds, int n, int64_t S, double* u) {
    for (int64_t s = 0; s < S; ++s)
        for (int k = 0; k < n; ++k) u[s * n + k] = oracle_uniform((uint64_t)seeds[k], s);
}

/* ------------------------------------------------------------------ the two precisions */

#define REAL double
#define SFX _f64
#include "oracle_impl.h"
#undef REAL
#undef SFX

#define REAL long double
#define SFX _ld
#include "oracle_impl.h"
#undef REAL
#undef SFX

/* ------------------------------------------------------------------ exported entry points */

int oracle_maxn(void) { return ORACLE_MAXN; }

/* Cofactors of one block: B [K1][K] complex128 (interleaved), rows [K1] the chosen output modes
 * of its rows (equal ids = equal rows).  P [K] complex.  Returns the addend count.  */
int64_t oracle_cofactors_f64(const double* B, const int64_t* rows, int K1, int K, double* P) {
    init_binom();
    if (K1 < 0 || K > ORACLE_MAXN || K != K1 + 1) return -1;
    return cofactors_f64(B, rows, K1, K, P);
}

/* Same in x87 extended precision; B and P stay float64 at the interface.  */
int64_t oracle_cofactors_ld(const double* B, const int64_t* rows, int K1, int K, double* P) {
    init_binom();
    if (K1 < 0 || K > ORACLE_MAXN || K != K1 + 1) return -1;
    long double Bl[2 * ORACLE_MAXN * ORACLE_MAXN], Pl[2 * ORACLE_MAXN];
    for (int i = 0; i < 2 * K1 * K; ++i) Bl[i] = B[i];
    int64_t T = cofactors_ld(Bl, rows, K1, K, Pl);
    for (int c = 0; c < 2 * K; ++c) P[c] = (double)Pl[c];
    return T;
}

/* Addend count of one step (the closed form `variants.addends("2020", rows, cols)`).  */
int64_t oracle_addends(const int64_t* rows, int K1) {
    if (K1 == 0) return 1;
    int64_t drow[ORACLE_MAXN], N; int mult[ORACLE_MAXN], radix[ORACLE_MAXN]; double scale;
    tables_f64(rows, K1, drow, mult, radix, &N, &scale);
    return N;
}

/* One step: weights w [m] (unnormalised), returns the pick; gap as in step().  A [m][n] complex.  */
int64_t oracle_step_f64(const double* A, int m, int n, const int64_t* rows, const int64_t* cols, int k,
                        double u, double* w, double* gap) {
    init_binom();
    if (k < 1 || k > n || n > ORACLE_MAXN) return -1;
    return step_f64(A, m, n, rows, cols, k, u, w, gap, NULL);
}

int64_t oracle_step_ld(const double* A, int m, int n, const int64_t* rows, const int64_t* cols, int k,
                       double u, double* w, double* gap) {
    init_binom();
    if (k < 1 || k > n || n > ORACLE_MAXN) return -1;
    size_t na = (size_t)m * (size_t)n * 2;
    long double* Al = (long double*)malloc(sizeof(long double) * na);
    long double* wl = (long double*)malloc(sizeof(long double) * (size_t)m);
    for (size_t i = 0; i < na; ++i) Al[i] = A[i];
    int64_t r = step_ld(Al, m, n, rows, cols, k, u, wl, gap, NULL);
    if (w) for (int i = 0; i < m; ++i) w[i] = (double)wl[i];
    free(Al); free(wl);
    return r;
}

/* Streams are handed to `threads` POSIX threads through an atomic counter (dynamic schedule). */
typedef struct {
    int ld;                       /* 0: double, 1: long double */
    const double* A; const long double* Al; int m, n, steps;
    const int64_t* dp; const int64_t* sigma; const double* u; int64_t S;
    int64_t* rows; double* marg; double* gap; int64_t* addends;
    atomic_llong next;
} chain_job;

static void* chain_worker(void* arg) {
    chain_job* J = (chain_job*)arg;
    size_t inst = (size_t)J->m * J->n * 2;
    long double* ml = NULL;
    if (J->ld && J->marg) ml = (long double*)malloc(sizeof(long double) * (size_t)J->steps * J->m);
    for (;;) {
        int64_t s = atomic_fetch_add(&J->next, 1);
        if (s >= J->S) break;
        if (!J->ld) {
            chain_one_f64(J->A + (size_t)J->dp[s] * inst, J->m, J->n, J->steps, J->sigma + s * J->steps,
                          J->u + s * J->steps, J->rows + s * J->steps,
                          J->marg ? J->marg + (size_t)s * J->steps * J->m : NULL,
                          J->gap ? J->gap + s * J->steps : NULL, J->addends ? J->addends + s : NULL);
        } else {
            chain_one_ld(J->Al + (size_t)J->dp[s] * inst, J->m, J->n, J->steps, J->sigma + s * J->steps,
                         J->u + s * J->steps, J->rows + s * J->steps, ml,
                         J->gap ? J->gap + s * J->steps : NULL, J->addends ? J->addends + s : NULL);
            if (ml) for (size_t i = 0; i < (size_t)J->steps * J->m; ++i) J->marg[(size_t)s * J->steps * J->m + i] = (double)ml[i];
        }
    }
    free(ml);
    return NULL;
}

static int run_chain(chain_job* J, int threads) {
    if (threads <= 0) { long c = sysconf(_SC_NPROCESSORS_ONLN); threads = c > 0 ? (int)c : 1; }
    if (threads > 256) threads = 256;
    atomic_init(&J->next, 0);
    pthread_t tid[256];
    int started = 0;
    for (int i = 1; i < threads; ++i) if (pthread_create(&tid[started], NULL, chain_worker, J) == 0) ++started;
    chain_worker(J);
    for (int i = 0; i < started; ++i) pthread_join(tid[i], NULL);
    return 0;
}

/* Whole chains of S streams of `steps` photons each (FP64), parallel over streams with `threads` host
 * threads (<= 0: all online cores).  A [G][m][n] complex128, dp [S], sigma [S][steps] (column
 * indices < n), u [S][steps] -> rows [S][steps]; marg [S][steps][m] (w / tot), gap [S][steps] and
 * addends [S] are optional (NULL).  Returns 0, or -1 on bad sizes or indices.  */
static int check_chain_args(int G, int m, int n, int steps, const int64_t* dp, const int64_t* sigma, int64_t S) {
    if (n < 1 || n > ORACLE_MAXN || steps < 1 || steps > n || m < 1 || G < 1) return -1;
    for (int64_t s = 0; s < S; ++s) {
        if (dp[s] < 0 || dp[s] >= G) return -1;
        for (int k = 0; k < steps; ++k) if (sigma[s * steps + k] < 0 || sigma[s * steps + k] >= n) return -1;
    }
    return 0;
}

int oracle_chain_f64(const double* A, int G, int m, int n, int steps, const int64_t* dp, const int64_t* sigma,
                     const double* u, int64_t S, int64_t* rows, double* marg, double* gap,
                     int64_t* addends, int threads) {
    init_binom();
    if (check_chain_args(G, m, n, steps, dp, sigma, S)) return -1;
    chain_job J = {0, A, NULL, m, n, steps, dp, sigma, u, S, rows, marg, gap, addends, 0};
    return run_chain(&J, threads);
}

/* Same chain in x87 extended precision (marg returned as float64).  */
int oracle_chain_ld(const double* A, int G, int m, int n, int steps, const int64_t* dp, const int64_t* sigma,
                    const double* u, int64_t S, int64_t* rows, double* marg, double* gap,
                    int64_t* addends, int threads) {
    init_binom();
    if (check_chain_args(G, m, n, steps, dp, sigma, S)) return -1;
    size_t na = (size_t)G * m * n * 2;
    long double* Al = (long double*)malloc(sizeof(long double) * na);
    for (size_t i = 0; i < na; ++i) Al[i] = A[i];
    chain_job J = {1, NULL, Al, m, n, steps, dp, sigma, u, S, rows, marg, gap, addends, 0};
    int r = run_chain(&J, threads);
    free(Al);
    return r;
}
