// Clifford & Clifford exact Fock sampler for B200 (sm_100a): one persistent kernel runs whole
// chains, one CTA per stream at a time (a work queue hands out streams), everything of a step in
// shared memory and registers:
//
//   plan     thread 0: multiplicity tables of the chosen rows, halving rule, term count, and the
//            split of the collapsed Gray sum into CTA-uniform inner blocks, middle blocks and lanes
//   prepare  all threads: gather B = A[chosen rows, sigma(1..k)] into shared memory, fill the inner
//            Gray schedule (digit, sign, exact weight per term)
//   sweep    every Gray lane walks its terms; the row flipped at a term is the same for the whole
//            CTA (broadcast shared-memory reads, no divergence); all-but-one products by prefix and
//            suffix chains, split over TPL threads per lane; deterministic warp/CTA reduction
//   draw     marginal over all m output modes (coalesced column reads), FP64 block scan, inverse
//            CDF pick with the reference's rule, Philox uniforms identical to the reference's
//
// FP64 form: complex FP64 throughout.  Mixed form: inner blocks in complex FP32 (column sums
// re-initialised from FP64 at every block start), block sums folded into FP64 accumulators, FP64
// cross-lane reduction, marginal and CDF; a draw that falls within a guard band of a CDF step is
// recomputed with the FP64 sweep, so the mixed form picks what the FP64 form picks.
//
// Reference behaviour (Quandela/photonic-engines, file:line):
//   multiplicity tables / halving   photonic_engines/clifford/cofactors_triton.py:413-447
//   collapsed Gray sum              photonic_engines/clifford/cofactors_triton.py:141-260, cuda_cofactors.py:35-151
//   draw (scale, amplitudes, pick)  photonic_engines/clifford/cofactors_triton.py:263-309
//   step loop                       photonic_engines/clifford/sampler.py:391-460
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "pe_b200.h"
#include "pe_device.cuh"

namespace pe {

struct ChainParams {
    const double2* acol;
    const int64_t* inst_off;
    const int32_t* inst_m;
    const int32_t* inst_n;
    int G;
    int64_t S;
    const int64_t* dp;
    const int32_t* nk;
    const int64_t* cols;
    int n_stride;
    const double* uniforms;
    const int64_t* seeds;
    const int64_t* seed_row;
    const int64_t* rng_off;
    const int64_t* order;
    int64_t* rows;
    int64_t* occ;
    int occ_stride;
    double* marg;
    int marg_stride;
    unsigned long long* queue;
    int* status;
    long long* detail;
    int m_cap;
    double tau;     // mixed form: relative guard band of the draw
};

// Workspace layout: [0] queue counter (u64), [8] status (i32), [16] detail (i64).  Zeroed per call.
constexpr size_t WS_BYTES = 256;

static __device__ __forceinline__ void record_error(int* status, long long* detail, int64_t s) {
    if (atomicCAS(status, 0, PE_ERR_DEVICE) == 0) *detail = (long long)s;
}

// ---------------------------------------------------------------------------------------- plan
// Thread 0.  Multiplicity tables exactly as the reference builds them (sort, group, move the last
// odd group to the top slot, radix = mult + 1, top radix halved when an odd group exists), then
// the kernel's own enumeration split.  The order in which digits are enumerated does not change
// the sum; only the set of radices (hence N) is the reference's.
static __device__ void plan_step(Plan& pl, const int* rows, int K1, int K, int lanes) {
    int rs[MAXN];
    for (int i = 0; i < K1; ++i) rs[i] = rows[i];
    for (int i = 1; i < K1; ++i) {
        const int x = rs[i];
        int j = i - 1;
        while (j >= 0 && rs[j] > x) { rs[j + 1] = rs[j]; --j; }
        rs[j + 1] = x;
    }
    int drow[MAXN], mult[MAXN], radix[MAXN];
    int D = 0;
    for (int i = 0; i < K1; ++i) {
        if (D > 0 && drow[D - 1] == rs[i]) mult[D - 1]++;
        else { drow[D] = rs[i]; mult[D] = 1; ++D; }
    }
    int pos = -1;
    for (int q = 0; q < D; ++q) if (mult[q] & 1) pos = q;
    if (pos >= 0 && pos != D - 1) {
        int t = drow[pos]; drow[pos] = drow[D - 1]; drow[D - 1] = t;
        t = mult[pos]; mult[pos] = mult[D - 1]; mult[D - 1] = t;
    }
    int64_t N = 1;
    for (int q = 0; q < D; ++q) {
        radix[q] = (q == D - 1 && pos >= 0) ? (mult[q] + 1) / 2 : mult[q] + 1;
        N *= radix[q];
    }
    // active digits (radix >= 2) by ascending radix; radix-1 digits are fixed
    int act[MAXN], na = 0, fix[MAXN], nf = 0;
    for (int q = 0; q < D; ++q) {
        if (radix[q] >= 2) {
            int j = na++;
            while (j > 0 && radix[act[j - 1]] > radix[q]) { act[j] = act[j - 1]; --j; }
            act[j] = q;
        } else {
            fix[nf++] = q;
        }
    }
    // high digits: the prefix of `act` whose product best fills the lanes
    int nhi = na;
    int64_t H = N;
    if (N > lanes) {
        double best = -1.0;
        int64_t prod = 1;
        nhi = 1;
        for (int i = 0; i < na; ++i) {
            prod *= radix[act[i]];
            if (i > 0 && N / prod < 4) break;
            const double e = prod >= lanes
                ? (double)prod / ((double)lanes * (double)((prod + lanes - 1) / lanes))
                : (double)prod / (double)lanes;
            if (e > best + 1e-12) { best = e; nhi = i + 1; }
            if (prod >= lanes && e >= 0.95) break;
        }
        H = 1;
        for (int i = 0; i < nhi; ++i) H *= radix[act[i]];
    }
    // inner: leading low digits while the block fits the schedule table; the rest are middle
    int nin = 0, Lin = 1;
    while (nhi + nin < na && Lin * radix[act[nhi + nin]] <= LIN_MAX) { Lin *= radix[act[nhi + nin]]; ++nin; }
    const int nmid = na - nhi - nin;
    int64_t Lmid = 1;
    int kd = 0;
    for (int i = 0; i < nin; ++i, ++kd) { const int q = act[nhi + i]; pl.R[kd] = radix[q]; pl.M[kd] = mult[q]; pl.drow[kd] = drow[q]; }
    for (int i = 0; i < nmid; ++i, ++kd) { const int q = act[nhi + nin + i]; pl.R[kd] = radix[q]; pl.M[kd] = mult[q]; pl.drow[kd] = drow[q]; Lmid *= radix[q]; }
    for (int i = 0; i < nhi; ++i, ++kd) { const int q = act[i]; pl.R[kd] = radix[q]; pl.M[kd] = mult[q]; pl.drow[kd] = drow[q]; }
    for (int i = 0; i < nf; ++i, ++kd) { const int q = fix[i]; pl.R[kd] = 1; pl.M[kd] = mult[q]; pl.drow[kd] = drow[q]; }
    pl.N = N; pl.H = H; pl.Lmid = Lmid; pl.Lin = Lin;
    pl.K = K; pl.K1 = K1; pl.D = D;
    pl.nin = nin; pl.nmid = nmid; pl.nhi = nhi;
    pl.scale = (pos >= 0 ? 2.0 : 1.0) * ldexp(1.0, -K1);
}

// ---------------------------------------------------------------------------------------- prepare
// All threads.  Element (rho, j) of the instance is A[rho * rs + j * cs].
static __device__ void prepare_step(Smem& sm, const double2* __restrict__ A, int64_t rs, int64_t cs, bool mixed) {
    const Plan& pl = sm.plan;
    const int tid = threadIdx.x, T = blockDim.x;
    for (int idx = tid; idx < pl.D * MAXN; idx += T) {
        const int kd = idx / MAXN, j = idx % MAXN;
        double2 b = make_double2(0.0, 0.0);
        if (j < pl.K) b = A[(int64_t)pl.drow[kd] * rs + (int64_t)sm.cols[j] * cs];
        sm.B[kd][j] = b;
        if (mixed) sm.B32[kd][j] = make_float2((float)(2.0 * b.x), (float)(2.0 * b.y));
    }
    const int nin = pl.nin;
    for (int t = tid; t < pl.Lin; t += T) {
        int d[MAXN], v[MAXN];
        int rem = t;
        for (int q = 0; q < nin; ++q) { d[q] = rem % pl.R[q]; rem /= pl.R[q]; }
        int par = 0;
        for (int q = nin - 1; q >= 0; --q) { v[q] = (par & 1) ? pl.R[q] - 1 - d[q] : d[q]; par += v[q]; }
        double w = 1.0;
        for (int q = 0; q < nin; ++q) w *= signed_binom(pl.M[q], v[q]);
        sm.tab_w[t] = w;
        sm.tab_w32[t] = (float)w;
        unsigned char e = 0;
        if (t > 0) {
            int q = 0;
            while (d[q] == 0) ++q;                       // the digit the odometer moved
            int parh = 0;
            for (int mu = q + 1; mu < nin; ++mu) parh += v[mu];
            const int dir = (parh & 1) ? -1 : 1;         // v_q moved by dir: column sums move by -2 dir b_q
            e = (unsigned char)(q | (dir > 0 ? 0x80 : 0));
        }
        sm.tab_f[t] = e;
        if (t == pl.Lin - 1)
            for (int q = 0; q < nin; ++q) sm.plan.vend[q] = (unsigned char)v[q];
    }
}

// ---------------------------------------------------------------------------------------- sweep
// acc_c += w * prod_{j != c} s_j over this thread's KH columns; the other TPL - 1 threads of the
// lane contribute the product of their columns (exchanged once per term).  w enters the prefix
// chain of the lane's first thread.
template <int KH, int TPL, typename R>
__device__ __forceinline__ void allbutone_acc(const R (&sr)[KH], const R (&si)[KH], R w, R (&ar)[KH], R (&ai)[KH],
                                              int h, unsigned gmask) {
    R pr[KH], pi[KH];
    R xr = (h == 0) ? w : R(1), xi = R(0);
#pragma unroll
    for (int c = 0; c < KH; ++c) {
        pr[c] = xr; pi[c] = xi;
        const R nr = xr * sr[c] - xi * si[c];
        xi = xr * si[c] + xi * sr[c];
        xr = nr;
    }
    R yr, yi;
    if constexpr (TPL == 1) {
        yr = R(1); yi = R(0);
    } else if constexpr (TPL == 2) {
        yr = __shfl_xor_sync(gmask, xr, 1);
        yi = __shfl_xor_sync(gmask, xi, 1);
    } else {
        const R qr = __shfl_xor_sync(gmask, xr, 1), qi = __shfl_xor_sync(gmask, xi, 1);
        const R pr2 = xr * qr - xi * qi, pi2 = xr * qi + xi * qr;
        const R orr = __shfl_xor_sync(gmask, pr2, 2), oi = __shfl_xor_sync(gmask, pi2, 2);
        yr = qr * orr - qi * oi;
        yi = qr * oi + qi * orr;
    }
#pragma unroll
    for (int c = KH - 1; c >= 0; --c) {
        ar[c] += pr[c] * yr - pi[c] * yi;
        ai[c] += pr[c] * yi + pi[c] * yr;
        const R nr = yr * sr[c] - yi * si[c];
        yi = yr * si[c] + yi * sr[c];
        yr = nr;
    }
}

// Deterministic reduction of the per-thread accumulators over the lanes of the CTA -> sm.P.
template <int KH, int TPL>
__device__ __forceinline__ void reduce_to_P(double (&ar)[KH], double (&ai)[KH], Smem& sm, int c0) {
    const int tid = threadIdx.x, lid = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int j = 0; j < KH; ++j) {
#pragma unroll
        for (int o = TPL; o < 32; o <<= 1) {
            ar[j] += __shfl_xor_sync(0xffffffffu, ar[j], o);
            ai[j] += __shfl_xor_sync(0xffffffffu, ai[j], o);
        }
    }
    if (lid < TPL) {
#pragma unroll
        for (int j = 0; j < KH; ++j) sm.red[wid][c0 + j] = make_double2(ar[j], ai[j]);
    }
    __syncthreads();
    if (tid < sm.plan.K) {
        double xr = 0.0, xi = 0.0;
        for (int w = 0; w < nw; ++w) { xr += sm.red[w][tid].x; xi += sm.red[w][tid].y; }
        sm.P[tid] = make_double2(xr * sm.plan.scale, xi * sm.plan.scale);
    }
    __syncthreads();
}

template <int TPL>
__device__ __forceinline__ unsigned group_mask() {
    if constexpr (TPL == 1) return 0u;
    else return ((1u << TPL) - 1u) << ((threadIdx.x & 31) & ~(TPL - 1));
}

// FP64 sweep of tier KP (columns padded to KP: padded column sums hold 1, their B rows are zero).
template <int KP, int TPL>
__device__ void sweep_f64(Smem& sm) {
    constexpr int KH = KP / TPL;
    const Plan& pl = sm.plan;
    const int tid = threadIdx.x, T = blockDim.x;
    const int lanes = T / TPL, lane = tid / TPL, h = tid % TPL, c0 = h * KH;
    const unsigned gmask = group_mask<TPL>();
    const int nin = pl.nin, nmid = pl.nmid, nhi = pl.nhi, D = pl.D, K = pl.K, Lin = pl.Lin;
    const int64_t Lmid = pl.Lmid, H = pl.H;
    double ar[KH], ai[KH];
#pragma unroll
    for (int j = 0; j < KH; ++j) { ar[j] = 0.0; ai[j] = 0.0; }
    for (int64_t hl = lane; hl < H; hl += lanes) {
        double sr[KH], si[KH];
#pragma unroll
        for (int j = 0; j < KH; ++j) { sr[j] = 0.0; si[j] = 0.0; }
        double wh = 1.0;
        int64_t rem = hl;
        for (int kd = 0; kd < D; ++kd) {
            int v = 0;
            if (kd >= nin + nmid && kd < nin + nmid + nhi) {
                v = (int)(rem % pl.R[kd]);
                rem /= pl.R[kd];
                wh *= signed_binom(pl.M[kd], v);
            }
            const double c = (double)(pl.M[kd] - 2 * v);
            const double2* b = &sm.B[kd][c0];
#pragma unroll
            for (int j = 0; j < KH; ++j) { sr[j] = fma(c, b[j].x, sr[j]); si[j] = fma(c, b[j].y, si[j]); }
        }
#pragma unroll
        for (int j = 0; j < KH; ++j) if (c0 + j >= K) { sr[j] = 1.0; si[j] = 0.0; }
        unsigned char dm[MAXN], vm[MAXN], pp[MAXN];
        for (int q = 0; q < nmid; ++q) { dm[q] = 0; vm[q] = 0; pp[q] = 0; }
        double wm = 1.0;
        for (int64_t pm = 0; pm < Lmid; ++pm) {
            if (pm > 0) {
                int q = 0;
                while (dm[q] == pl.R[nin + q] - 1) ++q;
                const int dir = pp[q] ? -1 : 1;
                for (int mu = 0; mu < q; ++mu) { dm[mu] = 0; pp[mu] ^= 1; }
                dm[q] += 1;
                vm[q] = (unsigned char)(vm[q] + dir);
                const double f = -2.0 * dir;
                const double2* b = &sm.B[nin + q][c0];
#pragma unroll
                for (int j = 0; j < KH; ++j) { sr[j] = fma(f, b[j].x, sr[j]); si[j] = fma(f, b[j].y, si[j]); }
                wm = 1.0;
                for (int mu = 0; mu < nmid; ++mu) wm *= signed_binom(pl.M[nin + mu], vm[mu]);
            }
            const double wmh = wh * wm;
            if (!(pm & 1)) {
                for (int t = 0; t < Lin; ++t) {
                    if (t > 0) {
                        const unsigned e = sm.tab_f[t];
                        const double f = (e & 0x80u) ? -2.0 : 2.0;
                        const double2* b = &sm.B[e & 63u][c0];
#pragma unroll
                        for (int j = 0; j < KH; ++j) { sr[j] = fma(f, b[j].x, sr[j]); si[j] = fma(f, b[j].y, si[j]); }
                    }
                    allbutone_acc<KH, TPL, double>(sr, si, wmh * sm.tab_w[t], ar, ai, h, gmask);
                }
            } else {
                for (int t = Lin - 1; t >= 0; --t) {
                    if (t < Lin - 1) {
                        const unsigned e = sm.tab_f[t + 1];
                        const double f = (e & 0x80u) ? 2.0 : -2.0;
                        const double2* b = &sm.B[e & 63u][c0];
#pragma unroll
                        for (int j = 0; j < KH; ++j) { sr[j] = fma(f, b[j].x, sr[j]); si[j] = fma(f, b[j].y, si[j]); }
                    }
                    allbutone_acc<KH, TPL, double>(sr, si, wmh * sm.tab_w[t], ar, ai, h, gmask);
                }
            }
        }
    }
    reduce_to_P<KH, TPL>(ar, ai, sm, c0);
}

// Mixed sweep: every inner block starts from column sums formed in FP64 from the digit values
// (no drift carried across blocks), runs in complex FP32, and is folded into FP64 accumulators.
template <int KP, int TPL>
__device__ void sweep_mixed(Smem& sm) {
    constexpr int KH = KP / TPL;
    const Plan& pl = sm.plan;
    const int tid = threadIdx.x, T = blockDim.x;
    const int lanes = T / TPL, lane = tid / TPL, h = tid % TPL, c0 = h * KH;
    const unsigned gmask = group_mask<TPL>();
    const int nin = pl.nin, nmid = pl.nmid, nhi = pl.nhi, D = pl.D, K = pl.K, Lin = pl.Lin;
    const int64_t Lmid = pl.Lmid, H = pl.H;
    double ar[KH], ai[KH];
#pragma unroll
    for (int j = 0; j < KH; ++j) { ar[j] = 0.0; ai[j] = 0.0; }
    for (int64_t hl = lane; hl < H; hl += lanes) {
        unsigned char vh[MAXN];
        double wh = 1.0;
        {
            int64_t rem = hl;
            for (int i = 0; i < nhi; ++i) {
                const int kd = nin + nmid + i;
                const int v = (int)(rem % pl.R[kd]);
                rem /= pl.R[kd];
                vh[i] = (unsigned char)v;
                wh *= signed_binom(pl.M[kd], v);
            }
        }
        unsigned char dm[MAXN], vm[MAXN], pp[MAXN];
        for (int q = 0; q < nmid; ++q) { dm[q] = 0; vm[q] = 0; pp[q] = 0; }
        double wm = 1.0;
        for (int64_t pm = 0; pm < Lmid; ++pm) {
            if (pm > 0) {
                int q = 0;
                while (dm[q] == pl.R[nin + q] - 1) ++q;
                const int dir = pp[q] ? -1 : 1;
                for (int mu = 0; mu < q; ++mu) { dm[mu] = 0; pp[mu] ^= 1; }
                dm[q] += 1;
                vm[q] = (unsigned char)(vm[q] + dir);
                wm = 1.0;
                for (int mu = 0; mu < nmid; ++mu) wm *= signed_binom(pl.M[nin + mu], vm[mu]);
            }
            const bool fwd = !(pm & 1);
            float sr[KH], si[KH];
            {
                double xr[KH], xi[KH];
#pragma unroll
                for (int j = 0; j < KH; ++j) { xr[j] = 0.0; xi[j] = 0.0; }
                for (int kd = 0; kd < D; ++kd) {
                    int v = 0;
                    if (kd < nin) v = fwd ? 0 : sm.plan.vend[kd];
                    else if (kd < nin + nmid) v = vm[kd - nin];
                    else if (kd < nin + nmid + nhi) v = vh[kd - nin - nmid];
                    const double c = (double)(pl.M[kd] - 2 * v);
                    const double2* b = &sm.B[kd][c0];
#pragma unroll
                    for (int j = 0; j < KH; ++j) { xr[j] = fma(c, b[j].x, xr[j]); xi[j] = fma(c, b[j].y, xi[j]); }
                }
#pragma unroll
                for (int j = 0; j < KH; ++j) {
                    const bool pad = c0 + j >= K;
                    sr[j] = pad ? 1.0f : (float)xr[j];
                    si[j] = pad ? 0.0f : (float)xi[j];
                }
            }
            float a32r[KH], a32i[KH];
#pragma unroll
            for (int j = 0; j < KH; ++j) { a32r[j] = 0.0f; a32i[j] = 0.0f; }
            if (fwd) {
                for (int t = 0; t < Lin; ++t) {
                    if (t > 0) {
                        const unsigned e = sm.tab_f[t];
                        const float f = (e & 0x80u) ? -1.0f : 1.0f;
                        const float2* b = &sm.B32[e & 63u][c0];
#pragma unroll
                        for (int j = 0; j < KH; ++j) { sr[j] = fmaf(f, b[j].x, sr[j]); si[j] = fmaf(f, b[j].y, si[j]); }
                    }
                    allbutone_acc<KH, TPL, float>(sr, si, sm.tab_w32[t], a32r, a32i, h, gmask);
                }
            } else {
                for (int t = Lin - 1; t >= 0; --t) {
                    if (t < Lin - 1) {
                        const unsigned e = sm.tab_f[t + 1];
                        const float f = (e & 0x80u) ? 1.0f : -1.0f;
                        const float2* b = &sm.B32[e & 63u][c0];
#pragma unroll
                        for (int j = 0; j < KH; ++j) { sr[j] = fmaf(f, b[j].x, sr[j]); si[j] = fmaf(f, b[j].y, si[j]); }
                    }
                    allbutone_acc<KH, TPL, float>(sr, si, sm.tab_w32[t], a32r, a32i, h, gmask);
                }
            }
            const double wmh = wh * wm;
#pragma unroll
            for (int j = 0; j < KH; ++j) { ar[j] = fma(wmh, (double)a32r[j], ar[j]); ai[j] = fma(wmh, (double)a32i[j], ai[j]); }
        }
    }
    reduce_to_P<KH, TPL>(ar, ai, sm, c0);
}

#define PE_TIER(KPv, CALL)                                   \
    if constexpr (KPM >= KPv) {                              \
        if (K <= KPv) { CALL; return; }                      \
    }

template <int TPL, int KPM>
__device__ void dispatch_f64(Smem& sm, int K) {
    PE_TIER(4, (sweep_f64<4, TPL>(sm)))
    PE_TIER(8, (sweep_f64<8, TPL>(sm)))
    PE_TIER(12, (sweep_f64<12, TPL>(sm)))
    PE_TIER(16, (sweep_f64<16, TPL>(sm)))
    PE_TIER(20, (sweep_f64<20, TPL>(sm)))
    PE_TIER(24, (sweep_f64<24, TPL>(sm)))
    PE_TIER(28, (sweep_f64<28, TPL>(sm)))
    PE_TIER(32, (sweep_f64<32, TPL>(sm)))
}

template <int TPL, int KPM>
__device__ void dispatch_mixed(Smem& sm, int K) {
    PE_TIER(4, (sweep_mixed<4, TPL>(sm)))
    PE_TIER(8, (sweep_mixed<8, TPL>(sm)))
    PE_TIER(12, (sweep_mixed<12, TPL>(sm)))
    PE_TIER(16, (sweep_mixed<16, TPL>(sm)))
    PE_TIER(20, (sweep_mixed<20, TPL>(sm)))
    PE_TIER(24, (sweep_mixed<24, TPL>(sm)))
    PE_TIER(28, (sweep_mixed<28, TPL>(sm)))
    PE_TIER(32, (sweep_mixed<32, TPL>(sm)))
}

// ---------------------------------------------------------------------------------------- draw
// Marginal over the m output modes, FP64 block scan (contiguous chunk per thread, warp scan, warps
// in order), then idx = min(#{rho : cw_rho < u * tot}, m - 1) with tot = cw[m - 1]
// (cofactors_triton.py:298-308).  Returns the gap min |cw - u tot| / tot through sm.fmin[0].
static __device__ void draw_step(Smem& sm, double* __restrict__ wgt, const double2* __restrict__ A, int64_t rs, int64_t cs,
                          int m, int k, double u, double* __restrict__ marg_row) {
    const int tid = threadIdx.x, T = blockDim.x, lid = tid & 31, wid = tid >> 5, nw = T >> 5;
    for (int rho = tid; rho < m; rho += T) {
        double xr = 0.0, xi = 0.0;
        for (int c = 0; c < k; ++c) {
            const double2 a = A[(int64_t)rho * rs + (int64_t)sm.cols[c] * cs];
            const double2 p = sm.P[c];
            xr = fma(a.x, p.x, xr);
            xr = fma(-a.y, p.y, xr);
            xi = fma(a.x, p.y, xi);
            xi = fma(a.y, p.x, xi);
        }
        wgt[rho] = xr * xr + xi * xi;
    }
    __syncthreads();
    const int C = (m + T - 1) / T;
    const int lo = min(tid * C, m), hi = min(lo + C, m);
    double loc = 0.0;
    for (int i = lo; i < hi; ++i) loc += wgt[i];
    double x = loc;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double y = __shfl_up_sync(0xffffffffu, x, o);
        if (lid >= o) x += y;
    }
    double excl = __shfl_up_sync(0xffffffffu, x, 1);
    if (lid == 0) excl = 0.0;
    if (lid == 31) sm.scan[wid] = x;
    __syncthreads();
    double E = 0.0;
    for (int w = 0; w < wid; ++w) E += sm.scan[w];
    E += excl;
    if (lo <= m - 1 && m - 1 < hi) {
        double cw = E;
        for (int i = lo; i < hi; ++i) cw += wgt[i];
        sm.tot = cw;
        sm.target = u * cw;
    }
    __syncthreads();
    const double tot = sm.tot, target = sm.target;
    int cnt = 0;
    double gmin = 1.0e300;
    {
        double cw = E;
        for (int i = lo; i < hi; ++i) {
            cw += wgt[i];
            cnt += (cw < target) ? 1 : 0;
            gmin = fmin(gmin, fabs(cw - target));
        }
    }
    if (marg_row) for (int rho = tid; rho < m; rho += T) marg_row[rho] = wgt[rho] / tot;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        gmin = fmin(gmin, __shfl_xor_sync(0xffffffffu, gmin, o));
    }
    if (lid == 0) { sm.cnt[wid] = cnt; sm.fmin[wid] = gmin; }
    __syncthreads();
    if (tid == 0) {
        int c = 0;
        double g = 1.0e300;
        for (int w = 0; w < nw; ++w) { c += sm.cnt[w]; g = fmin(g, sm.fmin[w]); }
        sm.rows[k - 1] = min(c, m - 1);
        sm.fmin[0] = g / tot;
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------------------- chain
template <int TPL, int KPM, bool MIXED>
__device__ void chain_one(const ChainParams& p, Smem& sm, double* wgt, int64_t s) {
    const int tid = threadIdx.x;
    const int64_t g = p.dp[s];
    bool ok = g >= 0 && g < p.G;
    int m = 0, nin = 0;
    int64_t off = 0;
    if (ok) { m = p.inst_m[g]; nin = p.inst_n[g]; off = p.inst_off[g]; }
    const int nk = p.nk ? p.nk[s] : p.n_stride;
    ok = ok && nk >= 0 && nk <= p.n_stride && nk <= KPM && m >= 1 && m <= p.m_cap && m <= p.occ_stride;
    if (ok && tid < nk) {
        const int64_t c = p.cols[s * p.n_stride + tid];
        if (c < 0 || c >= nin) atomicOr(&sm.bad, 1);
        else sm.cols[tid] = (int)c;
    }
    if (!ok && tid == 0) sm.bad = 1;
    __syncthreads();
    if (sm.bad) {
        if (tid == 0) record_error(p.status, p.detail, s);
        return;
    }
    const double2* A = p.acol + off;      // (rho, j) at A[j * m + rho]
    for (int k = 1; k <= nk; ++k) {
        const int K = k, K1 = k - 1;
        if (K1 == 0) {
            if (tid == 0) sm.P[0] = make_double2(1.0, 0.0);
            __syncthreads();
        } else {
            if (tid == 0) plan_step(sm.plan, sm.rows, K1, K, blockDim.x / TPL);
            __syncthreads();
            prepare_step(sm, A, 1, m, MIXED);
            __syncthreads();
            if constexpr (MIXED) dispatch_mixed<TPL, KPM>(sm, K);
            else dispatch_f64<TPL, KPM>(sm, K);
        }
        double u;
        if (p.uniforms) {
            u = p.uniforms[s * p.n_stride + (k - 1)];
        } else {
            const int64_t row = p.seed_row ? p.seed_row[s] : 0;
            const int64_t ro = p.rng_off ? p.rng_off[s] : s;
            u = chain_uniform((uint64_t)p.seeds[row * p.n_stride + (k - 1)], ro);
        }
        double* mrow = p.marg ? p.marg + ((size_t)s * p.n_stride + (k - 1)) * p.marg_stride : nullptr;
        draw_step(sm, wgt, A, 1, m, m, k, u, mrow);
        if constexpr (MIXED) {
            if (K1 > 0 && sm.fmin[0] <= p.tau) {          // uniform: read after the draw's final barrier
                dispatch_f64<4, KPM>(sm, K);
                draw_step(sm, wgt, A, 1, m, m, k, u, mrow);
            }
        }
    }
    for (int j = tid; j < nk; j += blockDim.x) p.rows[s * p.n_stride + j] = sm.rows[j];
    if (p.occ) {
        for (int rho = tid; rho < p.occ_stride; rho += blockDim.x) {
            int c = 0;
            for (int j = 0; j < nk; ++j) c += (sm.rows[j] == rho) ? 1 : 0;
            p.occ[s * (int64_t)p.occ_stride + rho] = c;
        }
    }
}

__host__ __device__ constexpr size_t smem_fixed_bytes() { return (sizeof(Smem) + 15) & ~(size_t)15; }

template <int TPL, int KPM, bool MIXED>
__global__ void __launch_bounds__(256) fock_chain_kernel(ChainParams p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem& sm = *reinterpret_cast<Smem*>(smem_raw);
    double* wgt = reinterpret_cast<double*>(smem_raw + smem_fixed_bytes());
    const int tid = threadIdx.x;
    for (;;) {
        if (tid == 0) {
            const unsigned long long q = atomicAdd(p.queue, 1ull);
            sm.cur = (q < (unsigned long long)p.S) ? (p.order ? p.order[q] : (int64_t)q) : -1;
            sm.bad = 0;
        }
        __syncthreads();
        const int64_t s = sm.cur;
        if (s < 0) return;
        if (s >= p.S) {
            if (tid == 0) record_error(p.status, p.detail, s);
            return;
        }
        chain_one<TPL, KPM, MIXED>(p, sm, wgt, s);
        __syncthreads();
    }
}

// Cofactors of S independent blocks: A [S][m][K] row-major, rows [S][K - 1].
template <int TPL, int KPM, bool MIXED>
__global__ void __launch_bounds__(256) cofactor_kernel(const double2* __restrict__ A, const int64_t* __restrict__ rows,
                                                       int64_t S, int m, int K, double2* __restrict__ P,
                                                       int* status, long long* detail) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem& sm = *reinterpret_cast<Smem*>(smem_raw);
    const int tid = threadIdx.x;
    for (int64_t s = blockIdx.x; s < S; s += gridDim.x) {
        if (tid == 0) sm.bad = 0;
        __syncthreads();
        if (tid < K) sm.cols[tid] = tid;
        if (tid < K - 1) {
            const int64_t r = rows[s * (K - 1) + tid];
            if (r < 0 || r >= m) atomicOr(&sm.bad, 1);
            else sm.rows[tid] = (int)r;
        }
        __syncthreads();
        if (sm.bad) {
            if (tid == 0) record_error(status, detail, s);
            __syncthreads();
            continue;
        }
        if (K == 1) {
            if (tid == 0) sm.P[0] = make_double2(1.0, 0.0);
            __syncthreads();
        } else {
            if (tid == 0) plan_step(sm.plan, sm.rows, K - 1, K, blockDim.x / TPL);
            __syncthreads();
            prepare_step(sm, A + s * (int64_t)m * K, K, 1, MIXED);
            __syncthreads();
            if constexpr (MIXED) dispatch_mixed<TPL, KPM>(sm, K);
            else dispatch_f64<TPL, KPM>(sm, K);
        }
        if (tid < K) P[s * K + tid] = sm.P[tid];
        __syncthreads();
    }
}

}  // namespace pe
