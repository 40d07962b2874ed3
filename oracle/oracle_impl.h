/*
 * Body of the CPU oracle, instantiated twice by fock_oracle.c: once with REAL = double (the FP64
 * oracle, also the timed CPU baseline) and once with REAL = long double (x87 extended precision,
 * the error reference for the mixed-precision form).  TEST INFRASTRUCTURE ONLY: nothing in the
 * product path may call it.
 *
 * Restates, for one stream on the CPU:
 *   - the multiplicity tables of the chosen rows        photonic_engines/clifford/cofactors_triton.py:413-447
 *   - the reflected mixed-radix Gray sweep (odometer)    photonic_engines/clifford/cuda_cofactors.py:72-106
 *   - all-but-one products, exact (no division)          photonic_engines/clifford/variants.py:70-77
 *   - cofactor scale, amplitude contraction, pick rule   photonic_engines/clifford/cofactors_triton.py:287-308
 *   - the chain over steps k = 1..n                      photonic_engines/clifford/sampler.py:420-456
 *
 * The caller defines REAL, SFX (symbol suffix) before including this file.
 */

#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(name, SFX)

/* Per-step tables of K1 chosen rows (cofactors_triton.py:413-447): sort, group equal rows, move the
 * LAST odd-multiplicity group to the top slot (swap), radix = mult + 1, the top radix halved to
 * (mult + 1) / 2 when an odd group exists; scale = 2^-K1 (x2 when halved).  Returns D.  */
static int FN(tables)(const int64_t* rows, int K1, int64_t* drow, int* mult, int* radix,
                      int64_t* nterms, REAL* scale) {
    int64_t rs[ORACLE_MAXN];
    for (int i = 0; i < K1; ++i) rs[i] = rows[i];
    for (int i = 1; i < K1; ++i) {            /* insertion sort, ascending */
        int64_t x = rs[i]; int j = i - 1;
        while (j >= 0 && rs[j] > x) { rs[j + 1] = rs[j]; --j; }
        rs[j + 1] = x;
    }
    int D = 0;
    for (int i = 0; i < K1; ++i) {
        if (D > 0 && drow[D - 1] == rs[i]) mult[D - 1]++;
        else { drow[D] = rs[i]; mult[D] = 1; ++D; }
    }
    int pos = -1;
    for (int q = 0; q < D; ++q) if (mult[q] & 1) pos = q;      /* the last odd group */
    if (pos >= 0 && pos != D - 1) {
        int64_t tr = drow[pos]; drow[pos] = drow[D - 1]; drow[D - 1] = tr;
        int tm = mult[pos]; mult[pos] = mult[D - 1]; mult[D - 1] = tm;
    }
    int64_t N = 1;
    for (int q = 0; q < D; ++q) {
        radix[q] = (q == D - 1 && pos >= 0) ? (mult[q] + 1) / 2 : mult[q] + 1;
        N *= radix[q];
    }
    *nterms = N;
    *scale = (pos >= 0 ? (REAL)2 : (REAL)1) * (REAL)ldexp(1.0, -K1);
    return D;
}

/* prod_{j != c} s_j for every c, exactly (prefix and suffix products, no division), times w,
 * accumulated into acc.  Same quantity as variants.py:70-77 (explicit products).  */
static void FN(accum_allbutone)(const REAL* sr, const REAL* si, int K, REAL w, REAL* ar, REAL* ai) {
    REAL pr[ORACLE_MAXN], pi[ORACLE_MAXN];
    REAL xr = w, xi = 0;
    for (int c = 0; c < K; ++c) {
        pr[c] = xr; pi[c] = xi;
        REAL nr = xr * sr[c] - xi * si[c];
        xi = xr * si[c] + xi * sr[c];
        xr = nr;
    }
    REAL yr = 1, yi = 0;
    for (int c = K - 1; c >= 0; --c) {
        ar[c] += pr[c] * yr - pi[c] * yi;
        ai[c] += pr[c] * yi + pi[c] * yr;
        REAL nr = yr * sr[c] - yi * si[c];
        yi = yr * si[c] + yi * sr[c];
        yr = nr;
    }
}

/* Cofactors P_c = per(B \ column c) of the K1 x K block B (rows given in chosen order, repeats
 * allowed): the 2020 sum over v in prod_nu {0..R_nu - 1} walked by the reflected mixed-radix Gray
 * code of cuda_cofactors.py:72-106 (one digit moves by +-1 per term: s_j += -2 dirn b_nu,j).
 * The weight prod_nu (-1)^v_nu C(M_nu, v_nu) is recomputed exactly from the digits at every term
 * (the reference updates it by ratios).  B is [K1][K] complex, interleaved re/im.
 * Returns the number of addends (N).  */
static int64_t FN(cofactors)(const REAL* B, const int64_t* rows, int K1, int K, REAL* P) {
    if (K1 == 0) {
        for (int c = 0; c < K; ++c) { P[2 * c] = 1; P[2 * c + 1] = 0; }
        return 1;
    }
    int64_t drow[ORACLE_MAXN], N; int mult[ORACLE_MAXN], radix[ORACLE_MAXN]; REAL scale;
    int D = FN(tables)(rows, K1, drow, mult, radix, &N, &scale);
    /* distinct rows b_nu = the first row of B whose chosen mode is drow[nu] */
    REAL br[ORACLE_MAXN][ORACLE_MAXN], bi[ORACLE_MAXN][ORACLE_MAXN];
    for (int nu = 0; nu < D; ++nu) {
        int i = 0; while (rows[i] != drow[nu]) ++i;
        for (int j = 0; j < K; ++j) { br[nu][j] = B[2 * (i * K + j)]; bi[nu][j] = B[2 * (i * K + j) + 1]; }
    }
    unsigned char d[ORACLE_MAXN], v[ORACLE_MAXN], pp[ORACLE_MAXN];
    for (int nu = 0; nu < D; ++nu) { d[nu] = 0; v[nu] = 0; pp[nu] = 0; }
    REAL sr[ORACLE_MAXN], si[ORACLE_MAXN], ar[ORACLE_MAXN], ai[ORACLE_MAXN];
    for (int j = 0; j < K; ++j) { sr[j] = 0; si[j] = 0; ar[j] = 0; ai[j] = 0; }
    for (int nu = 0; nu < D; ++nu)
        for (int j = 0; j < K; ++j) { sr[j] += (REAL)mult[nu] * br[nu][j]; si[j] += (REAL)mult[nu] * bi[nu][j]; }
    for (int64_t t = 0; t < N; ++t) {
        if (t > 0) {
            int nu = 0;
            while (d[nu] == radix[nu] - 1) ++nu;
            int dirn = pp[nu] ? -1 : 1;
            for (int mu = 0; mu < nu; ++mu) { d[mu] = 0; pp[mu] ^= 1; }
            d[nu] += 1; v[nu] = (unsigned char)(v[nu] + dirn);
            REAL f = (REAL)(-2 * dirn);
            for (int j = 0; j < K; ++j) { sr[j] += f * br[nu][j]; si[j] += f * bi[nu][j]; }
        }
        REAL w = 1;
        for (int nu = 0; nu < D; ++nu) {
            REAL b = (REAL)binom_tab[mult[nu]][v[nu]];
            w *= (v[nu] & 1) ? -b : b;
        }
        FN(accum_allbutone)(sr, si, K, w, ar, ai);
    }
    for (int c = 0; c < K; ++c) { P[2 * c] = ar[c] * scale; P[2 * c + 1] = ai[c] * scale; }
    return N;
}

/* One chain step of one stream: candidate weights w[rho] = |sum_c A[rho, cols_c] P_c|^2 for every
 * rho < m, their running sum cw, and the pick idx = min(#{rho : cw_rho < u * tot}, m - 1)
 * (cofactors_triton.py:287-308; tot = cw[m-1], a sequential sum).  A is [m][n] complex.
 * gap receives min_rho |cw_rho - u tot| / tot, the distance of the draw to the nearest CDF step.  */
static int64_t FN(step)(const REAL* A, int m, int n, const int64_t* rows, const int64_t* cols, int k,
                        double u, REAL* wout, double* gap, int64_t* addends) {
    int K1 = k - 1, K = k;
    REAL B[2 * ORACLE_MAXN * ORACLE_MAXN], P[2 * ORACLE_MAXN];
    for (int i = 0; i < K1; ++i)
        for (int j = 0; j < K; ++j) {
            B[2 * (i * K + j)] = A[2 * (rows[i] * n + cols[j])];
            B[2 * (i * K + j) + 1] = A[2 * (rows[i] * n + cols[j]) + 1];
        }
    int64_t T = FN(cofactors)(B, rows, K1, K, P);
    if (addends) *addends += T;
    REAL cw = 0;
    REAL* cws = (REAL*)malloc(sizeof(REAL) * (size_t)m);
    for (int r = 0; r < m; ++r) {
        REAL xr = 0, xi = 0;
        for (int c = 0; c < K; ++c) {
            REAL a_r = A[2 * (r * n + cols[c])], a_i = A[2 * (r * n + cols[c]) + 1];
            xr += a_r * P[2 * c] - a_i * P[2 * c + 1];
            xi += a_r * P[2 * c + 1] + a_i * P[2 * c];
        }
        REAL w = xr * xr + xi * xi;
        if (wout) wout[r] = w;
        cw += w;
        cws[r] = cw;
    }
    REAL tot = cws[m - 1];
    REAL target = (REAL)u * tot;
    int64_t idx = 0;
    double g = 1e300;
    for (int r = 0; r < m; ++r) {
        if (cws[r] < target) ++idx;
        double dd = fabs((double)(cws[r] - target)) / (double)tot;
        if (dd < g) g = dd;
    }
    if (idx > m - 1) idx = m - 1;
    if (gap) *gap = g;
    free(cws);
    return idx;
}

/* The whole chain of one stream: As [m][n] complex (the input columns of its instance), sig [n]
 * the column order, u [n] the per-step uniforms.  Writes rows [n] (ordered output modes) and
 * optionally marg [n][m] (normalised weights w / tot of every step), gap [n] and the addend total.
 * sampler.py:420-456 with the 2020 step at every k.  */
static void FN(chain_one)(const REAL* As, int m, int n, int steps, const int64_t* sig, const double* u,
                          int64_t* rs, REAL* marg, double* gap, int64_t* addends) {
    REAL* w = (REAL*)malloc(sizeof(REAL) * (size_t)m);
    int64_t add = 0;
    for (int k = 1; k <= steps; ++k) {
        double g;
        rs[k - 1] = FN(step)(As, m, n, rs, sig, k, u[k - 1], w, &g, &add);
        if (gap) gap[k - 1] = g;
        if (marg) {
            REAL tot = 0;
            for (int r = 0; r < m; ++r) tot += w[r];
            for (int r = 0; r < m; ++r) marg[(size_t)(k - 1) * m + r] = w[r] / tot;
        }
    }
    if (addends) *addends = add;
    free(w);
}

#undef FN
#undef CAT
#undef CAT2
