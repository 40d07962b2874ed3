// Emitter inputs (EmitterMPS, chi = 2): the matrix-cofactor step of the generalised Clifford chain rule
// on B200.  Per lane (a stream and one pure term of its reduced state) and per Glynn sign vector delta in
// {+1} x {-1, +1}^(k-2) of the k-1 chosen rows:
//   colsum_{j,l} = sum_i delta_i U[row_i, mode(j, l)]                   (column sums, Gray-updated)
//   G_j = sum_l colsum_{j,l} M_{j,l}                                     (2 x 2)
//   q_c = f^dag G_{k-1} ... G_{c+1}     (backward, row vectors)   p_c = G_{c-1} ... G_0 s0  (forward)
//   t_{c,l} += sign(delta) q_c M_{c,l} p_c                               (= Tr(M_{c,l} K_c))
// then amp(rho) = 2^-(k-2) sum_c sum_l U[rho, mode(c, l)] t_{c,l} for every output mode rho, and the
// stream's weight w(rho) = sum over its lanes of |amp(rho)|^2.  This is the reference's
// matrix_cofactor_weights (photonic_engines/clifford/emitter_reference.py:280-305) and the step of
// emitter_sampler.sample_torch (emitter_sampler.py:150-175), restated for one warp per lane (k <= 8) or
// one CTA per lane (longer chains, whose 2^(k-2) sign vectors are spread over the CTA's threads).
#include <cuda_runtime.h>
#include <stdint.h>

#include "pe_b200.h"
#include "pe_errors.h"

namespace pe_em {

constexpr int CHI = 2;
constexpr int THREADS = 128;
constexpr int NWARP = THREADS / 32;
constexpr int MAXK = 24;

struct Params {
    const double2* UT;          // [M][m]: UT[mode * m + rho] = U[rho, mode]
    int m, M;
    const int64_t* rows;        // [S][rows_stride]: the chosen rows, first k - 1 valid
    int rows_stride;
    const int32_t* colmode;     // [S][k][L]: input mode of label l of the stream's j-th slot (slots sorted)
    int64_t S;
    int k, L;
    const double2* s0;          // [Tt][2]
    const double2* f;           // [Tt][2]
    const double2* mats;        // [Tt][k][L][2][2]
    int64_t Tt;
    const int64_t* lane_term;   // [nl]
    const int64_t* lane_stream; // [nl]
    int64_t nl;
    double2* amp;               // [nl][m]
    int* status;
    long long* detail;
};

static __device__ __forceinline__ void record(int* status, long long* detail, int64_t x) {
    if (atomicCAS(status, 0, PE_ERR_DEVICE) == 0) *detail = (long long)x;
}
static __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, -(a.y * b.y)), fma(a.x, b.y, a.y * b.x));
}
static __device__ __forceinline__ double2 cmac(double2 acc, double2 a, double2 b) {   // acc + a b
    return make_double2(fma(a.x, b.x, fma(-a.y, b.y, acc.x)), fma(a.x, b.y, fma(a.y, b.x, acc.y)));
}


// The Gray-ordered walk over sign-vector indices [t0, t1) of one lane: column sums, backward chain
// (stored), forward chain and the trace accumulators acc[c][l] += sign * q_c M_{c,l} p_c.  M and the
// rows' U entries are read from shared memory (sM[c][l][a][b], sU[i][j][l]).
template <int KE, int NL>
__device__ __forceinline__ void walk(const double2 (*sM)[NL][CHI][CHI], const double2 (*sU)[KE][NL], int k,
                                     int64_t t0, int64_t t1, double2 s00, double2 s01, double2 fc0, double2 fc1,
                                     double2 (&acc)[KE][NL]) {
    const int kk = k - 1;
#pragma unroll
    for (int j = 0; j < KE; ++j)
#pragma unroll
        for (int l = 0; l < NL; ++l) acc[j][l] = make_double2(0.0, 0.0);
    if (t0 < t1) {
        double2 cs[KE][NL];
        uint64_t g = (uint64_t)(t0 ^ (t0 >> 1));
#pragma unroll
        for (int j = 0; j < KE; ++j)
#pragma unroll
            for (int l = 0; l < NL; ++l) {
                double2 x = make_double2(kk == 0 ? 1.0 : 0.0, 0.0);
                if (j < k) {
                    for (int i = 0; i < kk; ++i) {
                        const double d = (i == 0 || !((g >> (i - 1)) & 1)) ? 1.0 : -1.0;
                        x.x = fma(d, sU[i][j][l].x, x.x);
                        x.y = fma(d, sU[i][j][l].y, x.y);
                    }
                }
                cs[j][l] = x;
            }
        double sign = (__popcll(g) & 1) ? -1.0 : 1.0;
        for (int64_t t = t0; t < t1; ++t) {
            if (t > t0) {                                   // Gray step into t: free bit b flips
                const int b = __ffsll((long long)t) - 1;
                g ^= (uint64_t)1 << b;
                const double d2 = ((g >> b) & 1) ? -2.0 : 2.0;   // 2 * new delta of row b + 1
                const int i = b + 1;
#pragma unroll
                for (int j = 0; j < KE; ++j)
#pragma unroll
                    for (int l = 0; l < NL; ++l)
                        if (j < k) {
                            cs[j][l].x = fma(d2, sU[i][j][l].x, cs[j][l].x);
                            cs[j][l].y = fma(d2, sU[i][j][l].y, cs[j][l].y);
                        }
                sign = -sign;
            }
            // backward: q_c (stored), u <- u G_c
            double2 q0[KE], q1[KE];
            double2 u0 = fc0, u1 = fc1;
#pragma unroll
            for (int c = KE - 1; c >= 0; --c) {
                if (c < k) {
                    q0[c] = u0; q1[c] = u1;
                    double2 n0 = make_double2(0.0, 0.0), n1 = make_double2(0.0, 0.0);
#pragma unroll
                    for (int l = 0; l < NL; ++l) {
                        // z = u M_{c,l} (row vector), then u' += colsum z
                        const double2 z0 = cmac(cmul(u0, sM[c][l][0][0]), u1, sM[c][l][1][0]);
                        const double2 z1 = cmac(cmul(u0, sM[c][l][0][1]), u1, sM[c][l][1][1]);
                        n0 = cmac(n0, cs[c][l], z0);
                        n1 = cmac(n1, cs[c][l], z1);
                    }
                    u0 = n0; u1 = n1;
                }
            }
            // forward: y = M_{c,l} v, t_{c,l} += sign q_c . y, v <- sum_l colsum y
            double2 v0 = s00, v1 = s01;
#pragma unroll
            for (int c = 0; c < KE; ++c) {
                if (c < k) {
                    double2 n0 = make_double2(0.0, 0.0), n1 = make_double2(0.0, 0.0);
#pragma unroll
                    for (int l = 0; l < NL; ++l) {
                        const double2 y0 = cmac(cmul(sM[c][l][0][0], v0), sM[c][l][0][1], v1);
                        const double2 y1 = cmac(cmul(sM[c][l][1][0], v0), sM[c][l][1][1], v1);
                        const double2 dt = cmac(cmul(q0[c], y0), q1[c], y1);
                        acc[c][l].x = fma(sign, dt.x, acc[c][l].x);
                        acc[c][l].y = fma(sign, dt.y, acc[c][l].y);
                        n0 = cmac(n0, cs[c][l], y0);
                        n1 = cmac(n1, cs[c][l], y1);
                    }
                    v0 = n0; v1 = n1;
                }
            }
        }
    }
}

// The same walk with the stored backward chain and the trace accumulators in shared memory (too many
// values for registers at 16-24 columns): q[(c * 2 + a) * nt + t] and acc[(c * NL + l) * nt + t] for
// thread t of nt, consecutive threads at consecutive addresses.  The column sums stay in registers.
template <int KE, int NL>
__device__ __forceinline__ void walk_shared(const double2 (*sM)[NL][CHI][CHI], const double2 (*sU)[KE][NL], int k,
                                            int64_t t0, int64_t t1, double2 s00, double2 s01, double2 fc0,
                                            double2 fc1, double2* q, double2* acc, int t, int nt) {
    const int kk = k - 1;
    for (int j = 0; j < k * NL; ++j) acc[j * nt + t] = make_double2(0.0, 0.0);
    if (t0 >= t1) return;
    double2 cs[KE][NL];
    uint64_t g = (uint64_t)(t0 ^ (t0 >> 1));
#pragma unroll
    for (int j = 0; j < KE; ++j)
#pragma unroll
        for (int l = 0; l < NL; ++l) {
            double2 x = make_double2(kk == 0 ? 1.0 : 0.0, 0.0);
            if (j < k) {
                for (int i = 0; i < kk; ++i) {
                    const double d = (i == 0 || !((g >> (i - 1)) & 1)) ? 1.0 : -1.0;
                    x.x = fma(d, sU[i][j][l].x, x.x);
                    x.y = fma(d, sU[i][j][l].y, x.y);
                }
            }
            cs[j][l] = x;
        }
    double sign = (__popcll(g) & 1) ? -1.0 : 1.0;
    for (int64_t tt = t0; tt < t1; ++tt) {
        if (tt > t0) {
            const int b = __ffsll((long long)tt) - 1;
            g ^= (uint64_t)1 << b;
            const double d2 = ((g >> b) & 1) ? -2.0 : 2.0;
            const int i = b + 1;
#pragma unroll
            for (int j = 0; j < KE; ++j)
#pragma unroll
                for (int l = 0; l < NL; ++l)
                    if (j < k) {
                        cs[j][l].x = fma(d2, sU[i][j][l].x, cs[j][l].x);
                        cs[j][l].y = fma(d2, sU[i][j][l].y, cs[j][l].y);
                    }
            sign = -sign;
        }
        double2 u0 = fc0, u1 = fc1;
#pragma unroll
        for (int c = KE - 1; c >= 0; --c) {
            if (c < k) {
                q[(c * 2) * nt + t] = u0;
                q[(c * 2 + 1) * nt + t] = u1;
                double2 n0 = make_double2(0.0, 0.0), n1 = make_double2(0.0, 0.0);
#pragma unroll
                for (int l = 0; l < NL; ++l) {
                    const double2 z0 = cmac(cmul(u0, sM[c][l][0][0]), u1, sM[c][l][1][0]);
                    const double2 z1 = cmac(cmul(u0, sM[c][l][0][1]), u1, sM[c][l][1][1]);
                    n0 = cmac(n0, cs[c][l], z0);
                    n1 = cmac(n1, cs[c][l], z1);
                }
                u0 = n0; u1 = n1;
            }
        }
        double2 v0 = s00, v1 = s01;
#pragma unroll
        for (int c = 0; c < KE; ++c) {
            if (c < k) {
                const double2 qa = q[(c * 2) * nt + t], qb = q[(c * 2 + 1) * nt + t];
                double2 n0 = make_double2(0.0, 0.0), n1 = make_double2(0.0, 0.0);
#pragma unroll
                for (int l = 0; l < NL; ++l) {
                    const double2 y0 = cmac(cmul(sM[c][l][0][0], v0), sM[c][l][0][1], v1);
                    const double2 y1 = cmac(cmul(sM[c][l][1][0], v0), sM[c][l][1][1], v1);
                    const double2 dt = cmac(cmul(qa, y0), qb, y1);
                    double2& a = acc[(c * NL + l) * nt + t];
                    a.x = fma(sign, dt.x, a.x);
                    a.y = fma(sign, dt.y, a.y);
                    n0 = cmac(n0, cs[c][l], y0);
                    n1 = cmac(n1, cs[c][l], y1);
                }
                v0 = n0; v1 = n1;
            }
        }
    }
}

template <int KE, int NL>
__global__ void __launch_bounds__(THREADS) emitter_amp_kernel(Params p) {
    __shared__ double2 sM[KE][NL][CHI][CHI];
    __shared__ double2 sU[KE][KE][NL];          // sU[i][j][l] = U[row_i, mode(j, l)], i < k - 1
    __shared__ double2 red[NWARP][KE][NL];
    __shared__ double2 sT[KE][NL];
    __shared__ int sMode[KE][NL];
    __shared__ int sRow[KE];
    __shared__ int bad;
    const int tid = threadIdx.x, lid = tid & 31, wid = tid >> 5;
    const int k = p.k, kk = k - 1;
    for (int64_t lane = blockIdx.x; lane < p.nl; lane += gridDim.x) {
        if (tid == 0) bad = 0;
        __syncthreads();
        const int64_t s = p.lane_stream[lane], e = p.lane_term[lane];
        if (s < 0 || s >= p.S || e < 0 || e >= p.Tt) {
            if (tid == 0) record(p.status, p.detail, lane);
            __syncthreads();
            continue;
        }
        if (tid < k * NL) {
            const int j = tid / NL, l = tid % NL;
            const int md = p.colmode[(s * k + j) * p.L + l];
            if (md < 0 || md >= p.M) atomicOr(&bad, 1);
            else sMode[j][l] = md;
        }
        if (tid < kk) {
            const int64_t r = p.rows[s * p.rows_stride + tid];
            if (r < 0 || r >= p.m) atomicOr(&bad, 1);
            else sRow[tid] = (int)r;
        }
        for (int idx = tid; idx < k * NL * CHI * CHI; idx += THREADS) {
            const int j = idx / (NL * CHI * CHI), rem = idx % (NL * CHI * CHI);
            const int l = rem / (CHI * CHI), ab = rem % (CHI * CHI);
            sM[j][l][ab / CHI][ab % CHI] = p.mats[(e * k + j) * (int64_t)p.L * CHI * CHI + l * CHI * CHI + ab];
        }
        __syncthreads();
        if (bad) {
            if (tid == 0) record(p.status, p.detail, lane);
            __syncthreads();
            continue;
        }
        for (int idx = tid; idx < kk * k * NL; idx += THREADS) {
            const int i = idx / (k * NL), rem = idx % (k * NL);
            const int j = rem / NL, l = rem % NL;
            sU[i][j][l] = p.UT[(int64_t)sMode[j][l] * p.m + sRow[i]];
        }
        __syncthreads();
        const double2 s00 = p.s0[e * CHI], s01 = p.s0[e * CHI + 1];
        const double2 f0 = p.f[e * CHI], f1 = p.f[e * CHI + 1];
        const double2 fc0 = make_double2(f0.x, -f0.y), fc1 = make_double2(f1.x, -f1.y);

        // this thread's contiguous block [t0, t1) of Gray indices over the k - 2 free signs
        const int64_t D = kk >= 1 ? ((int64_t)1 << (kk - 1)) : 1;
        int64_t t0, t1;
        if (D >= THREADS) { const int64_t per = D / THREADS; t0 = tid * per; t1 = t0 + per; }
        else { t0 = tid; t1 = tid < D ? tid + 1 : tid; }
        double2 acc[KE][NL];
        walk<KE, NL>(sM, sU, k, t0, t1, s00, s01, fc0, fc1, acc);
        // deterministic reduction: warp butterflies, then the warps in order
#pragma unroll
        for (int j = 0; j < KE; ++j)
#pragma unroll
            for (int l = 0; l < NL; ++l) {
                double2 x = acc[j][l];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    x.x += __shfl_xor_sync(0xffffffffu, x.x, o);
                    x.y += __shfl_xor_sync(0xffffffffu, x.y, o);
                }
                if (lid == 0 && j < k) red[wid][j][l] = x;
            }
        __syncthreads();
        const double norm = kk >= 1 ? ldexp(1.0, -(kk - 1)) : 1.0;
        if (tid < k * NL) {
            const int j = tid / NL, l = tid % NL;
            double2 x = make_double2(0.0, 0.0);
            for (int w = 0; w < NWARP; ++w) { x.x += red[w][j][l].x; x.y += red[w][j][l].y; }
            sT[j][l] = make_double2(x.x * norm, x.y * norm);
        }
        __syncthreads();
        for (int rho = tid; rho < p.m; rho += THREADS) {
            double2 a = make_double2(0.0, 0.0);
            for (int c = 0; c < k; ++c)
#pragma unroll
                for (int l = 0; l < NL; ++l) a = cmac(a, p.UT[(int64_t)sMode[c][l] * p.m + rho], sT[c][l]);
            p.amp[lane * p.m + rho] = a;
        }
        __syncthreads();
    }
}

// Short chains (k <= 8: at most 64 sign vectors per lane): one warp per lane, eight lanes per CTA, each
// warp with its own slice of shared memory; no CTA barrier.
constexpr int WW = 8;
template <int NL>
__global__ void __launch_bounds__(32 * WW) emitter_amp_warp_kernel(Params p) {
    constexpr int KE = 8;
    __shared__ double2 wM[WW][KE][NL][CHI][CHI];
    __shared__ double2 wU[WW][KE][KE][NL];
    __shared__ double2 wT[WW][KE][NL];
    __shared__ int wMode[WW][KE][NL];
    __shared__ int wRow[WW][KE];
    const int lid = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int k = p.k, kk = k - 1;
    for (int64_t lane = (int64_t)blockIdx.x * WW + wid; lane < p.nl; lane += (int64_t)gridDim.x * WW) {
        const int64_t s = p.lane_stream[lane], e = p.lane_term[lane];
        const bool bad_lane = s < 0 || s >= p.S || e < 0 || e >= p.Tt;
        bool bad = false;
        if (!bad_lane && lid < k * NL) {
            const int j = lid / NL, l = lid % NL;
            const int md = p.colmode[(s * k + j) * p.L + l];
            if (md < 0 || md >= p.M) bad = true;
            else wMode[wid][j][l] = md;
        }
        if (!bad_lane && lid < kk) {
            const int64_t r = p.rows[s * p.rows_stride + lid];
            if (r < 0 || r >= p.m) bad = true;
            else wRow[wid][lid] = (int)r;
        }
        if (bad_lane || __any_sync(0xffffffffu, bad)) {
            if (lid == 0) record(p.status, p.detail, lane);
            __syncwarp();
            continue;
        }
        for (int idx = lid; idx < k * NL * CHI * CHI; idx += 32) {
            const int j = idx / (NL * CHI * CHI), rem = idx % (NL * CHI * CHI);
            const int l = rem / (CHI * CHI), ab = rem % (CHI * CHI);
            wM[wid][j][l][ab / CHI][ab % CHI] = p.mats[(e * k + j) * (int64_t)p.L * CHI * CHI + l * CHI * CHI + ab];
        }
        __syncwarp();
        for (int idx = lid; idx < kk * k * NL; idx += 32) {
            const int i = idx / (k * NL), rem = idx % (k * NL);
            const int j = rem / NL, l = rem % NL;
            wU[wid][i][j][l] = p.UT[(int64_t)wMode[wid][j][l] * p.m + wRow[wid][i]];
        }
        __syncwarp();
        const double2 s00 = p.s0[e * CHI], s01 = p.s0[e * CHI + 1];
        const double2 f0 = p.f[e * CHI], f1 = p.f[e * CHI + 1];
        const int64_t D = kk >= 1 ? ((int64_t)1 << (kk - 1)) : 1;
        int64_t t0, t1;
        if (D >= 32) { const int64_t per = D / 32; t0 = lid * per; t1 = t0 + per; }
        else { t0 = lid; t1 = lid < D ? lid + 1 : lid; }
        double2 acc[KE][NL];
        walk<KE, NL>(wM[wid], wU[wid], k, t0, t1, s00, s01, make_double2(f0.x, -f0.y), make_double2(f1.x, -f1.y), acc);
        const double norm = kk >= 1 ? ldexp(1.0, -(kk - 1)) : 1.0;
#pragma unroll
        for (int j = 0; j < KE; ++j)
#pragma unroll
            for (int l = 0; l < NL; ++l) {
                double2 x = acc[j][l];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    x.x += __shfl_xor_sync(0xffffffffu, x.x, o);
                    x.y += __shfl_xor_sync(0xffffffffu, x.y, o);
                }
                if (lid == 0 && j < k) wT[wid][j][l] = make_double2(x.x * norm, x.y * norm);
            }
        __syncwarp();
        for (int rho = lid; rho < p.m; rho += 32) {
            double2 a = make_double2(0.0, 0.0);
            for (int c = 0; c < k; ++c)
#pragma unroll
                for (int l = 0; l < NL; ++l) a = cmac(a, p.UT[(int64_t)wMode[wid][c][l] * p.m + rho], wT[wid][c][l]);
            p.amp[lane * p.m + rho] = a;
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------------------- fused step
// The same step with every term assembled on the device from the per-state tables: a lane is (stream s,
// term e < nlan[s]); its matrices are gathers of gops[a][b][r][l] = K^{(a,b)}_r M_{a,l} (the gap channel
// after placed slot a, Kraus operator r, times the slot's emission operator) and of ops for the last
// placed slot, its vectors rows of pre[a] (images of |s0>) and suf[fid][b] (images of <final|).  The term
// index decodes as (i0, if, g_0 .. g_{k-2}) with g_{k-2} fastest; a term whose norm is below 1e-14 of its
// scale contributes nothing (the rule of the host decomposition).
struct Tables {
    const double2* gops;     // [n][n][4][L][2][2]
    const int32_t* rg;       // [n][n]
    const double2* ops;      // [n][L][2][2]
    const double2* pre;      // [n][2][2]
    const int32_t* r0;       // [n]
    const double2* suf;      // [nf][n][2][2]
    const int32_t* rf;       // [nf][n]
    int n, nf;
};

struct StepParams {
    const double2* UT;
    int m, M;
    const int64_t* rows;
    int rows_stride;
    const int32_t* T;        // [S][k] placed slots, increasing
    const int32_t* fid;      // [S]
    const int32_t* modes;    // [n][L]
    int64_t S;
    int k, L;
    Tables tb;
    const int64_t* lstart;   // [S]
    const int64_t* nlan;     // [S]
    int64_t nl;
    double2* amp;            // [nl][m]
    int* status;
    long long* detail;
};

// nlan[s] = number of terms of stream s (0 and an error record for invalid slots / final ids).
__global__ void emitter_count_kernel(StepParams p, int64_t* nlan) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= p.S) return;
    const int32_t* T = p.T + s * p.k;
    const int fid = p.fid[s];
    bool ok = fid >= 0 && fid < p.tb.nf;
    int64_t R = 0;
    if (ok) {
        for (int j = 0; j < p.k; ++j) ok = ok && T[j] >= 0 && T[j] < p.tb.n && (j == 0 || T[j] > T[j - 1]);
    }
    if (ok) {
        R = (int64_t)p.tb.r0[T[0]] * p.tb.rf[fid * p.tb.n + T[p.k - 1]];
        for (int j = 0; j + 1 < p.k; ++j) R *= p.tb.rg[T[j] * p.tb.n + T[j + 1]];
    } else {
        record(p.status, p.detail, s);
    }
    nlan[s] = R;
}

// Stream of a lane: the last s with lstart[s] <= lane (binary search; empty streams share their
// successor's start, so the last one is the stream that owns the lane).
static __device__ __forceinline__ int64_t stream_of(const int64_t* lstart, int64_t S, int64_t lane) {
    int64_t lo = 0, hi = S - 1;
    while (lo < hi) {
        const int64_t mid = (lo + hi + 1) >> 1;
        if (lstart[mid] <= lane) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Load lane `lane` into the caller's shared arrays (one thread group of `nt` threads, thread index `t`,
// whose first warp holds threads 0..31): returns false (uniformly) when the lane is invalid or its term has
// zero norm.  Thread 0 decodes the term index into sG (gap choices) and sI (i0, if); the group gathers the
// matrices and vectors; lanes 0..3 of the first warp run the norm's transfer chain (one component each).
template <int KE, int NL>
__device__ bool load_fused(const StepParams& p, int64_t lane, int t, int nt, double2 (*sM)[NL][CHI][CHI],
                           double2 (*sU)[KE][NL], int (*sMode)[NL], int* sRow, double2* sS0, double2* sF, int* flag,
                           int* sG, bool warp) {
    const int k = p.k, kk = k - 1;
    const int64_t s = stream_of(p.lstart, p.S, lane);
    const int32_t* T = p.T + s * k;
    const int fid = p.fid[s];
    if (t == 0) {
        int ok = 1;
        int64_t e = lane - p.lstart[s];
        if (e < 0 || e >= p.nlan[s]) ok = 0;
        for (int j = k - 2; j >= 0 && ok; --j) {
            const int rk = p.tb.rg[T[j] * p.tb.n + T[j + 1]];
            sG[j] = (int)(e % rk);
            e /= rk;
        }
        if (ok) {
            const int rfv = p.tb.rf[fid * p.tb.n + T[k - 1]];
            sG[KE] = (int)(e / rfv);            // i0
            sG[KE + 1] = (int)(e % rfv);        // if
        }
        *flag = ok;
    }
    if (warp) __syncwarp(); else __syncthreads();
    if (!*flag) return false;
    for (int idx = t; idx < k * NL * CHI * CHI; idx += nt) {
        const int c = idx / (NL * CHI * CHI), rem = idx % (NL * CHI * CHI);
        const int l = rem / (CHI * CHI), ab = rem % (CHI * CHI);
        const double2* src = c + 1 < k
            ? p.tb.gops + ((((int64_t)T[c] * p.tb.n + T[c + 1]) * 4 + sG[c]) * p.L + l) * CHI * CHI
            : p.tb.ops + ((int64_t)T[c] * p.L + l) * CHI * CHI;
        sM[c][l][ab / CHI][ab % CHI] = src[ab];
    }
    if (t < 2) sS0[t] = p.tb.pre[((int64_t)T[0] * 2 + sG[KE]) * CHI + t];
    else if (t < 4) sF[t - 2] = p.tb.suf[(((int64_t)fid * p.tb.n + T[k - 1]) * 2 + sG[KE + 1]) * CHI + (t - 2)];
    if (warp) __syncwarp(); else __syncthreads();
    if (t < 32) {
        // norm^2 = <f (x) f*| E_{k-1} ... E_0 |s0 (x) s0*>, E_c = sum_l M_{c,l} (x) M_{c,l}*; lane j < 4 holds
        // component j = (t1, u1) of the transfer vector (lanes 4..31 compute a copy of component j % 4)
        const int j = t & 3, t1 = j >> 1, u1 = j & 1;
        double2 v = cmul(sS0[t1], make_double2(sS0[u1].x, -sS0[u1].y));
        for (int c = 0; c < k; ++c) {
            double2 vs[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                vs[q].x = __shfl_sync(0xffffffffu, v.x, (t & ~3) + q);
                vs[q].y = __shfl_sync(0xffffffffu, v.y, (t & ~3) + q);
            }
            double2 nv = make_double2(0.0, 0.0);
#pragma unroll
            for (int l = 0; l < NL; ++l)
#pragma unroll
                for (int s1 = 0; s1 < 2; ++s1)
#pragma unroll
                    for (int v1 = 0; v1 < 2; ++v1) {
                        const double2 mc = sM[c][l][u1][v1];
                        nv = cmac(nv, cmul(sM[c][l][t1][s1], make_double2(mc.x, -mc.y)), vs[s1 * 2 + v1]);
                    }
            v = nv;
        }
        const double2 w = cmul(make_double2(sF[t1].x, -sF[t1].y), sF[u1]);      // f_a* f_b
        double part = w.x * v.x - w.y * v.y;
        part += __shfl_xor_sync(0xffffffffu, part, 1);
        part += __shfl_xor_sync(0xffffffffu, part, 2);
        if (t == 0) {
            const double sc = (sF[0].x * sF[0].x + sF[0].y * sF[0].y + sF[1].x * sF[1].x + sF[1].y * sF[1].y) *
                              (sS0[0].x * sS0[0].x + sS0[0].y * sS0[0].y + sS0[1].x * sS0[1].x + sS0[1].y * sS0[1].y);
            if (!(part > 1e-14 * (sc > 1.0 ? sc : 1.0))) *flag = 0;
        }
    }
    if (warp) __syncwarp(); else __syncthreads();
    if (!*flag) return false;
    int bad = 0;
    if (t < k * NL) {
        const int jj = t / NL, l = t % NL;
        const int md = p.modes[T[jj] * p.L + l];
        if (md < 0 || md >= p.M) bad = 1;
        else sMode[jj][l] = md;
    }
    if (t < kk) {
        const int64_t r = p.rows[s * p.rows_stride + t];
        if (r < 0 || r >= p.m) bad = 1;
        else sRow[t] = (int)r;
    }
    if (bad) { atomicOr(flag, 2); record(p.status, p.detail, lane); }
    if (warp) __syncwarp(); else __syncthreads();
    if (*flag & 2) return false;
    for (int idx = t; idx < kk * k * NL; idx += nt) {
        const int i = idx / (k * NL), rem = idx % (k * NL);
        const int jj = rem / NL, l = rem % NL;
        sU[i][jj][l] = p.UT[(int64_t)sMode[jj][l] * p.m + sRow[i]];
    }
    if (warp) __syncwarp(); else __syncthreads();
    return true;
}

template <int NL>
__global__ void __launch_bounds__(32 * WW) emitter_step_warp_kernel(StepParams p) {
    constexpr int KE = 8;
    __shared__ double2 wM[WW][KE][NL][CHI][CHI];
    __shared__ double2 wU[WW][KE][KE][NL];
    __shared__ double2 wT[WW][KE][NL];
    __shared__ double2 wS0[WW][2], wF[WW][2];
    __shared__ int wMode[WW][KE][NL];
    __shared__ int wRow[WW][KE];
    __shared__ int wFlag[WW];
    __shared__ int wG[WW][KE + 2];
    const int lid = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int k = p.k, kk = k - 1;
    for (int64_t lane = (int64_t)blockIdx.x * WW + wid; lane < p.nl; lane += (int64_t)gridDim.x * WW) {
        if (!load_fused<KE, NL>(p, lane, lid, 32, wM[wid], wU[wid], wMode[wid], wRow[wid], wS0[wid], wF[wid],
                                &wFlag[wid], wG[wid], true)) {
            for (int rho = lid; rho < p.m; rho += 32) p.amp[lane * p.m + rho] = make_double2(0.0, 0.0);
            __syncwarp();
            continue;
        }
        const int64_t D = kk >= 1 ? ((int64_t)1 << (kk - 1)) : 1;
        int64_t t0, t1;
        if (D >= 32) { const int64_t per = D / 32; t0 = lid * per; t1 = t0 + per; }
        else { t0 = lid; t1 = lid < D ? lid + 1 : lid; }
        double2 acc[KE][NL];
        walk<KE, NL>(wM[wid], wU[wid], k, t0, t1, wS0[wid][0], wS0[wid][1], make_double2(wF[wid][0].x, -wF[wid][0].y),
                     make_double2(wF[wid][1].x, -wF[wid][1].y), acc);
        const double norm = kk >= 1 ? ldexp(1.0, -(kk - 1)) : 1.0;
#pragma unroll
        for (int j = 0; j < KE; ++j)
#pragma unroll
            for (int l = 0; l < NL; ++l) {
                double2 x = acc[j][l];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    x.x += __shfl_xor_sync(0xffffffffu, x.x, o);
                    x.y += __shfl_xor_sync(0xffffffffu, x.y, o);
                }
                if (lid == 0 && j < k) wT[wid][j][l] = make_double2(x.x * norm, x.y * norm);
            }
        __syncwarp();
        for (int rho = lid; rho < p.m; rho += 32) {
            double2 a = make_double2(0.0, 0.0);
            for (int c = 0; c < k; ++c)
#pragma unroll
                for (int l = 0; l < NL; ++l) a = cmac(a, p.UT[(int64_t)wMode[wid][c][l] * p.m + rho], wT[wid][c][l]);
            p.amp[lane * p.m + rho] = a;
        }
        __syncwarp();
    }
}

constexpr int STHREADS = 64;          // threads per lane of the wide fused step (more sign vectors each)
template <int KE, int NL>
__host__ __device__ constexpr size_t step_dyn_smem() { return (size_t)STHREADS * (2 * KE + KE * NL) * sizeof(double2); }

template <int KE, int NL>
__global__ void __launch_bounds__(STHREADS) emitter_step_kernel(StepParams p) {
    extern __shared__ __align__(16) unsigned char dyn[];
    double2* q = reinterpret_cast<double2*>(dyn);                  // [2 KE][STHREADS]
    double2* acc = q + 2 * KE * STHREADS;                           // [KE NL][STHREADS]
    __shared__ double2 sM[KE][NL][CHI][CHI];
    __shared__ double2 sU[KE][KE][NL];
    __shared__ double2 sT[KE][NL];
    __shared__ double2 sS0[2], sF[2];
    __shared__ int sMode[KE][NL];
    __shared__ int sRow[KE];
    __shared__ int flag;
    __shared__ int sG[KE + 2];
    const int tid = threadIdx.x;
    const int k = p.k, kk = k - 1;
    for (int64_t lane = blockIdx.x; lane < p.nl; lane += gridDim.x) {
        if (!load_fused<KE, NL>(p, lane, tid, STHREADS, sM, sU, sMode, sRow, sS0, sF, &flag, sG, false)) {
            for (int rho = tid; rho < p.m; rho += STHREADS) p.amp[lane * p.m + rho] = make_double2(0.0, 0.0);
            __syncthreads();
            continue;
        }
        const int64_t D = kk >= 1 ? ((int64_t)1 << (kk - 1)) : 1;
        int64_t t0, t1;
        if (D >= STHREADS) { const int64_t per = D / STHREADS; t0 = tid * per; t1 = t0 + per; }
        else { t0 = tid; t1 = tid < D ? tid + 1 : tid; }
        walk_shared<KE, NL>(sM, sU, k, t0, t1, sS0[0], sS0[1], make_double2(sF[0].x, -sF[0].y),
                            make_double2(sF[1].x, -sF[1].y), q, acc, tid, STHREADS);
        __syncthreads();
        const double norm = kk >= 1 ? ldexp(1.0, -(kk - 1)) : 1.0;
        if (tid < k * NL) {                                       // threads in order: deterministic
            double2 x = make_double2(0.0, 0.0);
            for (int w = 0; w < STHREADS; ++w) { const double2 a = acc[tid * STHREADS + w]; x.x += a.x; x.y += a.y; }
            sT[tid / NL][tid % NL] = make_double2(x.x * norm, x.y * norm);
        }
        __syncthreads();
        for (int rho = tid; rho < p.m; rho += STHREADS) {
            double2 a = make_double2(0.0, 0.0);
            for (int c = 0; c < k; ++c)
#pragma unroll
                for (int l = 0; l < NL; ++l) a = cmac(a, p.UT[(int64_t)sMode[c][l] * p.m + rho], sT[c][l]);
            p.amp[lane * p.m + rho] = a;
        }
        __syncthreads();
    }
}

template <int KE, int NL>
static int launch_step_wide(const StepParams& p, cudaStream_t st) {
    const size_t dyn = step_dyn_smem<KE, NL>();
    PE_CUDA_TRY(cudaFuncSetAttribute(emitter_step_kernel<KE, NL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    PE_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, emitter_step_kernel<KE, NL>, STHREADS, dyn));
    if (per < 1) return PE_ERR_SIZE;
    int64_t grid = (int64_t)sms * per;
    if (grid > p.nl) grid = p.nl;
    emitter_step_kernel<KE, NL><<<(unsigned)grid, STHREADS, dyn, st>>>(p);
    return ::pe::launch_status();
}

template <class K>
static int occupancy_grid(K kernel, int threads, int64_t units, int64_t* grid) {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    PE_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, 0));
    if (per < 1) return PE_ERR_SIZE;
    *grid = (int64_t)sms * per;
    if (*grid > units) *grid = units;
    if (*grid < 1) *grid = 1;
    return PE_OK;
}

template <int NL>
static int launch_amp_warp(const Params& p, cudaStream_t st) {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    PE_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, emitter_amp_warp_kernel<NL>, 32 * WW, 0));
    if (per < 1) return PE_ERR_SIZE;
    int64_t grid = (int64_t)sms * per;
    const int64_t need = (p.nl + WW - 1) / WW;
    if (grid > need) grid = need;
    emitter_amp_warp_kernel<NL><<<(unsigned)grid, 32 * WW, 0, st>>>(p);
    return ::pe::launch_status();
}

// w[s][rho] = sum over the stream's lanes lstart[s] .. lstart[s] + nlan[s] - 1, in order, of |amp|^2.
__global__ void emitter_weights_kernel(const double2* __restrict__ amp, const int64_t* __restrict__ lstart,
                                       const int64_t* __restrict__ nlan, int64_t S, int m, int64_t nl, double* w,
                                       int* status, long long* detail) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= S * m) return;
    const int64_t s = idx / m;
    const int rho = (int)(idx % m);
    const int64_t a = lstart[s], b = a + nlan[s];
    if (a < 0 || nlan[s] < 0 || b > nl) {
        if (rho == 0) record(status, detail, s);
        w[idx] = 0.0;
        return;
    }
    double x = 0.0;
    for (int64_t lane = a; lane < b; ++lane) {
        const double2 v = amp[lane * m + rho];
        x = fma(v.x, v.x, fma(v.y, v.y, x));
    }
    w[idx] = x;
}

template <int KE, int NL>
static int launch_amp(const Params& p, cudaStream_t st) {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    PE_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, emitter_amp_kernel<KE, NL>, THREADS, 0));
    if (per < 1) return PE_ERR_SIZE;
    int64_t grid = (int64_t)sms * per;
    if (grid > p.nl) grid = p.nl;
    emitter_amp_kernel<KE, NL><<<(unsigned)grid, THREADS, 0, st>>>(p);
    return ::pe::launch_status();
}

}  // namespace pe_em

using namespace pe_em;

extern "C" size_t pe_emitter_workspace_bytes(void) { return 256; }

extern "C" int pe_emitter_weights(const double* d_ut, int m, int M, const int64_t* d_rows, int rows_stride,
                                  const int32_t* d_colmode, int64_t S, int k, int L, int chi, const double* d_s0,
                                  const double* d_f, const double* d_mats, int64_t Tt, const int64_t* d_lane_term,
                                  const int64_t* d_lane_stream, const int64_t* d_lstart, const int64_t* d_nlan,
                                  int64_t nl, double* d_amp, double* d_w, void* d_workspace, size_t workspace_bytes,
                                  void* stream) {
    if (chi != CHI) return PE_ERR_SIZE;
    if (L < 1 || L > 2 || k < 1 || k > MAXK) return PE_ERR_SIZE;
    if (m < 1 || M < 1 || S < 0 || Tt < 0 || nl < 0 || rows_stride < (k > 1 ? k - 1 : 0)) return PE_ERR_ARG;
    if (!d_ut || !d_colmode || !d_s0 || !d_f || !d_mats || !d_lane_term || !d_lane_stream || !d_lstart || !d_nlan ||
        !d_amp || !d_w || !d_workspace || (k > 1 && !d_rows))
        return PE_ERR_ARG;
    if (workspace_bytes < 256) return PE_ERR_SIZE;
    cudaStream_t st = (cudaStream_t)stream;
    PE_CUDA_TRY(cudaMemsetAsync(d_workspace, 0, 256, st));
    if (S == 0) return PE_OK;
    Params p;
    p.UT = (const double2*)d_ut; p.m = m; p.M = M; p.rows = d_rows; p.rows_stride = rows_stride;
    p.colmode = d_colmode; p.S = S; p.k = k; p.L = L;
    p.s0 = (const double2*)d_s0; p.f = (const double2*)d_f; p.mats = (const double2*)d_mats; p.Tt = Tt;
    p.lane_term = d_lane_term; p.lane_stream = d_lane_stream; p.nl = nl; p.amp = (double2*)d_amp;
    p.status = (int*)((char*)d_workspace + 8);
    p.detail = (long long*)((char*)d_workspace + 16);
    int rc = PE_OK;
    if (nl > 0) {
        if (k <= 8) rc = L == 1 ? launch_amp_warp<1>(p, st) : launch_amp_warp<2>(p, st);
        else if (k <= 16) rc = L == 1 ? launch_amp<16, 1>(p, st) : launch_amp<16, 2>(p, st);
        else rc = L == 1 ? launch_amp<24, 1>(p, st) : launch_amp<24, 2>(p, st);
        if (rc != PE_OK) return rc;
    }
    const int64_t total = S * (int64_t)m;
    const int T = 256;
    emitter_weights_kernel<<<(unsigned)((total + T - 1) / T), T, 0, st>>>((const double2*)d_amp, d_lstart, d_nlan, S, m,
                                                                          nl, d_w, p.status, p.detail);
    return ::pe::launch_status();
}

extern "C" int pe_emitter_count(const int32_t* d_T, const int32_t* d_fid, int64_t S, int k, const int32_t* d_rg,
                                const int32_t* d_r0, const int32_t* d_rf, int n, int nf, int64_t* d_nlan,
                                void* d_workspace, size_t workspace_bytes, void* stream) {
    if (S < 0 || k < 1 || k > MAXK || n < 1 || k > n || nf < 1) return PE_ERR_SIZE;
    if (!d_T || !d_fid || !d_rg || !d_r0 || !d_rf || !d_nlan || !d_workspace) return PE_ERR_ARG;
    if (workspace_bytes < 256) return PE_ERR_SIZE;
    cudaStream_t st = (cudaStream_t)stream;
    PE_CUDA_TRY(cudaMemsetAsync(d_workspace, 0, 256, st));
    if (S == 0) return PE_OK;
    StepParams p = {};
    p.T = d_T; p.fid = d_fid; p.S = S; p.k = k;
    p.tb.rg = d_rg; p.tb.r0 = d_r0; p.tb.rf = d_rf; p.tb.n = n; p.tb.nf = nf;
    p.status = (int*)((char*)d_workspace + 8);
    p.detail = (long long*)((char*)d_workspace + 16);
    emitter_count_kernel<<<(unsigned)((S + 255) / 256), 256, 0, st>>>(p, d_nlan);
    return ::pe::launch_status();
}

extern "C" int pe_emitter_step(const double* d_ut, int m, int M, const int64_t* d_rows, int rows_stride,
                               const int32_t* d_T, const int32_t* d_fid, const int32_t* d_modes, int64_t S, int k,
                               int L, int chi, const double* d_gops, const int32_t* d_rg, const double* d_ops,
                               const double* d_pre, const int32_t* d_r0, const double* d_suf, const int32_t* d_rf,
                               int n, int nf, const int64_t* d_lstart, const int64_t* d_nlan, int64_t nl,
                               double* d_amp, double* d_w, void* d_workspace, size_t workspace_bytes, void* stream) {
    if (chi != CHI) return PE_ERR_SIZE;
    if (L < 1 || L > 2 || k < 1 || k > MAXK || n < 1 || k > n || nf < 1) return PE_ERR_SIZE;
    if (m < 1 || M < 1 || S < 0 || nl < 0 || rows_stride < (k > 1 ? k - 1 : 0)) return PE_ERR_ARG;
    if (!d_ut || !d_T || !d_fid || !d_modes || !d_gops || !d_rg || !d_ops || !d_pre || !d_r0 || !d_suf || !d_rf ||
        !d_lstart || !d_nlan || !d_amp || !d_w || !d_workspace || (k > 1 && !d_rows))
        return PE_ERR_ARG;
    if (workspace_bytes < 256) return PE_ERR_SIZE;
    cudaStream_t st = (cudaStream_t)stream;
    if (S == 0) return PE_OK;
    StepParams p;
    p.UT = (const double2*)d_ut; p.m = m; p.M = M; p.rows = d_rows; p.rows_stride = rows_stride;
    p.T = d_T; p.fid = d_fid; p.modes = d_modes; p.S = S; p.k = k; p.L = L;
    p.tb.gops = (const double2*)d_gops; p.tb.rg = d_rg; p.tb.ops = (const double2*)d_ops;
    p.tb.pre = (const double2*)d_pre; p.tb.r0 = d_r0; p.tb.suf = (const double2*)d_suf; p.tb.rf = d_rf;
    p.tb.n = n; p.tb.nf = nf;
    p.lstart = d_lstart; p.nlan = d_nlan; p.nl = nl; p.amp = (double2*)d_amp;
    p.status = (int*)((char*)d_workspace + 8);
    p.detail = (long long*)((char*)d_workspace + 16);
    int64_t grid = 0;
    int rc = PE_OK;
    if (nl > 0) {
        if (k <= 8) {
            if (L == 1) {
                if ((rc = occupancy_grid(emitter_step_warp_kernel<1>, 32 * WW, (nl + WW - 1) / WW, &grid)) != PE_OK) return rc;
                emitter_step_warp_kernel<1><<<(unsigned)grid, 32 * WW, 0, st>>>(p);
            } else {
                if ((rc = occupancy_grid(emitter_step_warp_kernel<2>, 32 * WW, (nl + WW - 1) / WW, &grid)) != PE_OK) return rc;
                emitter_step_warp_kernel<2><<<(unsigned)grid, 32 * WW, 0, st>>>(p);
            }
        } else if (k <= 16) {
            rc = L == 1 ? launch_step_wide<16, 1>(p, st) : launch_step_wide<16, 2>(p, st);
            if (rc != PE_OK) return rc;
        } else {
            rc = L == 1 ? launch_step_wide<24, 1>(p, st) : launch_step_wide<24, 2>(p, st);
            if (rc != PE_OK) return rc;
        }
        PE_CUDA_TRY(cudaGetLastError());
    }
    const int64_t total = S * (int64_t)m;
    emitter_weights_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>((const double2*)d_amp, d_lstart, d_nlan, S,
                                                                            m, nl, d_w, p.status, p.detail);
    return ::pe::launch_status();
}
