// Clifford & Clifford exact Fock sampler for B200 (sm_100a): one persistent kernel runs whole
// chains, one CTA per stream at a time (a work queue hands out streams), everything of a step in
// shared memory and registers:
//
//   plan     warp 0: radices of the collapsed sum from the chosen rows' multiplicities (kept
//            incrementally), halving rule, term count, and the split of the sum into CTA-uniform
//            inner blocks, middle blocks and Gray lanes
//   prepare  all threads: gather B = A[chosen rows, sigma(1..k)] into shared memory, fill the inner
//            and middle Gray schedules (digit, sign, exact weight per index)
//   sweep    every Gray lane walks its terms; the row flipped at a term is the same for the whole
//            CTA (broadcast shared-memory reads, no divergence); all-but-one products by prefix and
//            suffix chains, split over TPL threads per lane; deterministic warp/CTA reduction
//   draw     marginal over all m output modes (coalesced column reads), FP64 block scan, inverse
//            CDF pick with the reference's rule, Philox uniforms identical to the reference's
//
// FP64 form: complex FP64 throughout.  Mixed form: inner blocks in complex FP32 (column sums
// formed in FP64 at every block start), block sums folded into FP64 accumulators, FP64
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

#ifndef PE_UNROLL
#define PE_UNROLL 1         // Gray terms per inner-loop iteration (1 or 2)
#endif
#ifndef PE_SPLIT
#define PE_SPLIT 1          // FP64: split a thread's product chain in two interleaved halves (1-/2-thread lanes)
#endif
#ifndef PE_PAIR32
#define PE_PAIR32 1         // mixed form, 1- and 2-thread lanes: paired FP32 instructions (FFMA2 / FMUL2)
#endif
#ifndef PE_MAXT
#define PE_MAXT 256         // largest CTA the chain kernels are compiled for
#endif
#ifndef PE_MINB
#define PE_MINB 2           // resident PE_MAXT-thread CTAs per SM the register allocation must allow
#endif

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
    const int64_t* qrange;  // optional [2] on the device: the queue runs order[lo .. hi) only (a tier of a
                            // length-sorted batch); null: the whole [0, S)
    int64_t* rows;
    int64_t* occ;
    int occ_stride;
    double* marg;
    int marg_stride;
    unsigned long long* queue;
    int* status;
    long long* detail;
    int m_cap;
    double tau;     // mixed forms: relative guard band of the draw at a step of 20 columns ...
    double tau_log2g;  // ... growing by 2^tau_log2g per column (guard_band)
    int k_stop;     // run steps up to min(nk, k_stop) only (0: all); later steps go to the split kernels
    int64_t split_cap;  // with qrange: only queue positions below this stop at k_stop (the split kernels' slots);
                        // later positions run whole here.  -1: every stream stops at k_stop
    int k_first;    // first step to run (1: the whole chain); rows[s][0 .. k_first - 2] are given (a forced
                    // prefix, or the steps of an earlier launch).  A stream with nk < k_first - 1 is skipped.
};

// Mixed form: FP32 inner blocks of at most this many terms, each starting from FP64 column sums.
#ifndef PE_MIXED_LIN
#define PE_MIXED_LIN 512
#endif
constexpr int MIXED_LIN = PE_MIXED_LIN;

// Workspace layout: [0] queue counter (u64), [8] status (i32), [16] detail (i64).  Zeroed per call.
constexpr size_t WS_BYTES = 256;

static __device__ __forceinline__ void record_error(int* status, long long* detail, int64_t s);

// Guard band of a mixed form's draw at a step of k columns, relative to the total weight: a draw whose
// uniform lies closer than this to a CDF step is redone in FP64.  The FP32 sweeps' CDF deviation from
// FP64 grows geometrically with k, so the band does too.
static __device__ __forceinline__ double guard_band(const ChainParams& p, int k) {
    return p.tau * exp2((double)(k - 20) * p.tau_log2g);
}

// The stream that queue ticket q stands for: order[lo + q] over the range [lo, hi) of the queue (qrange,
// or the whole [0, S)); -1 once the range is drained.  An invalid range counts as empty and is recorded
// (detail S).
static __device__ __forceinline__ int64_t queue_stream(const ChainParams& p, unsigned long long q) {
    int64_t lo = 0, hi = p.S;
    if (p.qrange) {
        lo = p.qrange[0];
        hi = p.qrange[1];
        if (lo < 0 || hi > p.S || lo > hi) {
            if (q == 0) record_error(p.status, p.detail, p.S);
            return -1;
        }
    }
    const int64_t idx = lo + (int64_t)q;
    if (q >= (unsigned long long)(hi - lo)) return -1;
    return p.order ? p.order[idx] : idx;
}

static __device__ __forceinline__ void record_error(int* status, long long* detail, int64_t s) {
    if (atomicCAS(status, 0, PE_ERR_DEVICE) == 0) *detail = (long long)s;
}

// ---------------------------------------------------------------------------------------- groups
// Thread 0, after every pick: the distinct chosen modes and their multiplicities (the grouping of
// cofactors_triton.py:419-427, kept incrementally instead of re-sorting the rows every step).
template <class SM>
__device__ __forceinline__ void add_to_groups(SM& sm, int row) {
    for (int g = 0; g < sm.ngrp; ++g)
        if (sm.grow[g] == row) { sm.gmul[g] += 1; return; }
    sm.grow[sm.ngrp] = row;
    sm.gmul[sm.ngrp] = 1;
    sm.ngrp += 1;
}

// One whole warp: the groups of sm.rows[0, count) (count <= 32) in order of first appearance, as
// `count` calls of add_to_groups would leave them, in a few warp instructions: the lanes holding the
// same row find each other (match), the lowest of them leads, and leaders are numbered in lane order.
template <class SM>
__device__ __forceinline__ void build_groups_warp(SM& sm, int count) {
    const int lane = threadIdx.x & 31;
    if (count > 32) {                                          // chains beyond 33 photons: serial
        if (lane == 0) {
            sm.ngrp = 0;
            for (int i = 0; i < count; ++i) add_to_groups(sm, sm.rows[i]);
        }
        __syncwarp();
        return;
    }
    const bool has = lane < count;
    const int row = has ? sm.rows[lane] : -1 - lane;          // absent lanes: distinct non-rows
    const unsigned same = __match_any_sync(0xffffffffu, row);
    const bool leader = has && (__ffs(same) - 1 == lane);
    const unsigned leaders = __ballot_sync(0xffffffffu, leader);
    if (leader) {
        const int g = __popc(leaders & ((1u << lane) - 1u));
        sm.grow[g] = row;
        sm.gmul[g] = __popc(same);
    }
    if (lane == 0) sm.ngrp = __popc(leaders);
}

// ---------------------------------------------------------------------------------------- plan
// Value at rank position p (warp-uniform) of a per-lane array holding position lane + 32 q in [q].
template <int GL, typename T>
__device__ __forceinline__ T at_position(const T (&v)[GL], int p) {
    T x = v[0];
#pragma unroll
    for (int q = 1; q < GL; ++q)
        if (p >= 32 * q) x = v[q];
    return __shfl_sync(0xffffffffu, x, p & 31);
}

// Exclusive prefix product over rank positions (position lane + 32 q in [q]), in place.
template <int GL, typename T>
__device__ __forceinline__ void exclusive_product(T (&v)[GL]) {
    const int lane = threadIdx.x & 31;
    T carry = T(1);
#pragma unroll
    for (int q = 0; q < GL; ++q) {
        T x = v[q];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const T y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x *= y;
        }
        T ex = __shfl_up_sync(0xffffffffu, x, 1);
        if (lane == 0) ex = T(1);
        v[q] = ex * carry;
        carry *= __shfl_sync(0xffffffffu, x, 31);
    }
}

// Warp 0.  Lane g holds group g.  Radix = mult + 1, and one odd-multiplicity group (the last one)
// has its radix halved to (mult + 1) / 2 with the scale doubled — the complement symmetry
// v -> s - v of the reference (cofactors_triton.py:428-446); which odd group is halved does not
// change N or the sum.  Active digits (radix >= 2) are ranked by ascending radix (then group); the
// leading ones become the Gray lanes (best fill of the CTA's lanes), the next ones the inner block, then
// the middle block; what does not fit the schedules joins the lanes.  The ranking takes one ballot per
// distinct radix value, and every digit's table entries are written by the lane of its rank, so only
// the choice of the three splits walks the ranks one by one (in registers, read by shuffles).
template <class SM>
__device__ void plan_step(SM& sm, int K1, int K, int lanes, int lin_max, int mid_max) {
    auto& pl = sm.plan;
    constexpr int GL = (SM::NKMAX + 31) / 32;          // groups (and ranks) per lane: index lane + 32 q, q < GL
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    const int D = sm.ngrp;
    int halved = -1;                                   // the last group of odd multiplicity
#pragma unroll
    for (int q = 0; q < GL; ++q) {
        const int g = lane + 32 * q;
        const unsigned oddmask = __ballot_sync(full, g < D && (sm.gmul[g < D ? g : 0] & 1));
        if (oddmask) halved = 32 * q + 31 - __clz(oddmask);
    }
    int R[GL];
    bool active[GL];
#pragma unroll
    for (int q = 0; q < GL; ++q) {
        const int g = lane + 32 * q;
        const int M = g < D ? sm.gmul[g] : 0;
        R[q] = g < D ? (g == halved ? (M + 1) / 2 : M + 1) : 1;
        active[q] = R[q] >= 2;
    }
    // ranks by (radix, group): the groups of the smallest remaining radix take the next ranks in group order
    unsigned rem[GL];
#pragma unroll
    for (int q = 0; q < GL; ++q) rem[q] = __ballot_sync(full, active[q]);
    int na = 0;
    for (;;) {
        bool left = false;
#pragma unroll
        for (int q = 0; q < GL; ++q) left = left || rem[q] != 0u;
        if (!left) break;                              // warp-uniform: the masks are ballots
        int mine = 0x7fffffff;
#pragma unroll
        for (int q = 0; q < GL; ++q)
            if ((rem[q] >> lane) & 1u) mine = min(mine, R[q]);
        const int rmin = __reduce_min_sync(full, mine);
#pragma unroll
        for (int q = 0; q < GL; ++q) {
            const bool take = ((rem[q] >> lane) & 1u) && R[q] == rmin;
            const unsigned eq = __ballot_sync(full, take);
            if (take) {
                const int r = na + __popc(eq & below);
                pl.sortR[r] = R[q];
                pl.sortG[r] = lane + 32 * q;
            }
            na += __popc(eq);
            rem[q] &= ~eq;
        }
    }
    __syncwarp();
    long long rv[GL];                                  // radix at rank position lane + 32 q (1 past na)
#pragma unroll
    for (int q = 0; q < GL; ++q) rv[q] = lane + 32 * q < na ? pl.sortR[lane + 32 * q] : 1;
    long long pre[GL];                                 // product of the radices at positions <= p
#pragma unroll
    for (int q = 0; q < GL; ++q) pre[q] = rv[q];
    exclusive_product<GL>(pre);
#pragma unroll
    for (int q = 0; q < GL; ++q) pre[q] *= rv[q];
    const long long N = na > 0 ? at_position<GL>(pre, na - 1) : 1;
    // lanes: the prefix of the ranked digits that best fills the CTA's lanes
    int nhi = na;
    if (N > lanes) {
        double best = -1.0;
        nhi = 1;
        for (int i = 0; i < na; ++i) {
            const long long prod = at_position<GL>(pre, i);
            if (i > 0 && prod > N / 4) break;          // N / prod < 4
            const double e = prod >= lanes
                ? (double)prod / ((double)lanes * (double)((prod + lanes - 1) / lanes))
                : (double)prod / (double)lanes;
            if (e > best + 1e-12) { best = e; nhi = i + 1; }
            if (prod >= lanes && e >= 0.95) break;
        }
    }
    int nin = 0, Lin = 1;
    while (nhi + nin < na) {
        const int r = (int)at_position<GL>(rv, nhi + nin);
        if (Lin * r > lin_max) break;
        Lin *= r;
        ++nin;
    }
    int nmid = 0, Lmid = 1;
    while (nhi + nin + nmid < na) {
        const int r = (int)at_position<GL>(rv, nhi + nin + nmid);
        if (Lmid * r > mid_max) break;
        Lmid *= r;
        ++nmid;
    }
    // digit order: inner (kd 0..nin-1), middle, lanes, digits beyond both schedules (more lanes), then the
    // fixed digits (radix 1) in group order; Pin / Pmid the prefix products of the inner / middle radices
    int pin[GL], pmid[GL];
#pragma unroll
    for (int q = 0; q < GL; ++q) {
        const int p = lane + 32 * q;
        pin[q] = (p >= nhi && p < nhi + nin) ? (int)rv[q] : 1;
        pmid[q] = (p >= nhi + nin && p < nhi + nin + nmid) ? (int)rv[q] : 1;
    }
    exclusive_product<GL>(pin);
    exclusive_product<GL>(pmid);
    int nfix = 0;
#pragma unroll
    for (int q = 0; q < GL; ++q) {
        const int p = lane + 32 * q;
        if (p < na) {
            const int g = pl.sortG[p];
            const int kd = p < nhi ? nin + nmid + p : (p < nhi + nin + nmid ? p - nhi : p);
            pl.R[kd] = (int)rv[q];
            pl.M[kd] = sm.gmul[g];
            pl.drow[kd] = sm.grow[g];
            if (p >= nhi && p < nhi + nin) pl.Pin[kd] = pin[q];
            if (p >= nhi + nin && p < nhi + nin + nmid) pl.Pmid[kd - nin] = pmid[q];
        }
        const int g = lane + 32 * q;                   // fixed digits: after the active ones, in group order
        const bool fixed = g < D && !active[q];
        const unsigned fm = __ballot_sync(full, fixed);
        if (fixed) {
            const int kd = na + nfix + __popc(fm & below);
            pl.R[kd] = 1;
            pl.M[kd] = sm.gmul[g];
            pl.drow[kd] = sm.grow[g];
        }
        nfix += __popc(fm);
    }
    if (lane == 0) {
        pl.N = N; pl.H = N / ((long long)Lin * Lmid); pl.Lin = Lin; pl.Lmid = Lmid;
        pl.K = K; pl.K1 = K1; pl.D = D;
        pl.nin = nin; pl.nmid = nmid; pl.nhi = na - nin - nmid;
        pl.scale = (halved >= 0 ? 2.0 : 1.0) * ldexp(1.0, -K1);
    }
}

template <class PL>
static __device__ __forceinline__ unsigned char gray_entry(const PL& pl, int d0, int nd, const int* Pp, int t,
                                                          double* w_out, unsigned char* vend, bool binary) {
    if (binary) {                                   // every radix 2: the digits are the bits of t
        const int qstar = t > 0 ? __ffs(t) - 1 : -1;
        int par = 0, parh = 0;
        double w = 1.0;
        for (int q = nd - 1; q >= 0; --q) {
            if (q == qstar) parh = par;
            const int d = (t >> q) & 1;
            const int v = (par & 1) ? 1 - d : d;
            if (vend) vend[q] = (unsigned char)v;
            par += v;
            if (v) w *= -(double)pl.M[d0 + q];      // (-1)^v C(M, v) at v = 1
        }
        *w_out = w;
        if (qstar < 0) return 0;
        return (unsigned char)(qstar | ((parh & 1) ? 0 : 0x80));
    }
    int qstar = -1;
    if (t > 0) {
        for (int q = 0; q < nd; ++q)
            if ((t / Pp[q]) % pl.R[d0 + q] != 0) { qstar = q; break; }
    }
    int par = 0, parh = 0;
    double w = 1.0;
    for (int q = nd - 1; q >= 0; --q) {
        if (q == qstar) parh = par;
        const int R = pl.R[d0 + q];
        const int d = (t / Pp[q]) % R;
        const int v = (par & 1) ? R - 1 - d : d;
        if (vend) vend[q] = (unsigned char)v;
        par += v;
        w *= signed_binom(pl.M[d0 + q], v);
    }
    *w_out = w;
    if (qstar < 0) return 0;
    const int dir = (parh & 1) ? -1 : 1;            // v moved by dir: column sums move by -2 dir b
    return (unsigned char)(qstar | (dir > 0 ? 0x80 : 0));
}

// All threads.  Element (rho, j) of the instance is A[rho * rs + j * cs].  kh > 0 (mixed form with
// paired FP32 sweeps, kh columns per thread): row kd of B32 is written as float4 slots
// q = h * kh/2 + c holding (re b_j1, re b_j2, im b_j1, im b_j2) of 2b, j1 = h * kh + c, j2 = j1 + kh/2 —
// the two columns whose product chains one paired instruction advances together.
template <class SM>
static __device__ void prepare_step(SM& sm, const double2* __restrict__ A, int64_t rs, int64_t cs, bool mixed,
                                    int kh = 0) {
    constexpr int NK = SM::NKMAX;
    constexpr bool narrow = SM::NK32 == NK;           // the wide layout has no FP32 copy (FP64 only)
    const auto& pl = sm.plan;
    const int tid = threadIdx.x, T = blockDim.x;
    // the gather of B from L2: GB independent loads in flight per thread before any store (one L2 latency
    // per GB elements instead of one per element)
    constexpr int GB = 8;
    const int nel = pl.D * NK;
    for (int base = tid; base < nel; base += T * GB) {
        double2 v[GB];
#pragma unroll
        for (int g = 0; g < GB; ++g) {
            const int idx = base + g * T;
            const bool ok = idx < nel && idx % NK < pl.K;
            const int kd = ok ? idx / NK : 0, j = ok ? idx % NK : 0;      // in range even when not loaded
            v[g] = ok ? A[(int64_t)pl.drow[kd] * rs + (int64_t)sm.cols[j] * cs] : make_double2(0.0, 0.0);
        }
#pragma unroll
        for (int g = 0; g < GB; ++g) {
            const int idx = base + g * T;
            if (idx < nel) {
                const int kd = idx / NK, j = idx % NK;
                sm.B[kd][j] = v[g];
                if constexpr (narrow)
                    if (mixed && kh == 0) sm.B32[kd][j] = make_float2((float)(2.0 * v[g].x), (float)(2.0 * v[g].y));
            }
        }
    }
    if (narrow && mixed && kh > 0) {
        __syncthreads();
        const int ka = kh / 2;
        for (int idx = tid; idx < pl.D * (NK / 2); idx += T) {
            const int kd = idx / (NK / 2), q = idx % (NK / 2);
            const int j1 = (q / ka) * kh + q % ka, j2 = j1 + ka;
            const double2 b1 = j1 < pl.K ? sm.B[kd][j1] : make_double2(0.0, 0.0);
            const double2 b2 = j2 < pl.K ? sm.B[kd][j2] : make_double2(0.0, 0.0);
            reinterpret_cast<float4*>(&sm.B32[kd < SM::NK32 ? kd : 0][0])[q] =
                make_float4((float)(2.0 * b1.x), (float)(2.0 * b2.x), (float)(2.0 * b1.y), (float)(2.0 * b2.y));
        }
    }
    bool bin_in = true, bin_mid = true;             // schedules of radix-2 digits only (distinct rows)
    for (int q = 0; q < pl.nin; ++q) bin_in = bin_in && pl.R[q] == 2;
    for (int q = 0; q < pl.nmid; ++q) bin_mid = bin_mid && pl.R[pl.nin + q] == 2;
    for (int t = tid; t < pl.Lin; t += T) {
        double w;
        sm.tab_f[t] = gray_entry(pl, 0, pl.nin, pl.Pin, t, &w, t == pl.Lin - 1 ? sm.plan.vend : nullptr, bin_in);
        sm.tab_w[t] = w;
        sm.tab_w32[t] = (float)w;
    }
    for (int t = tid; t < pl.Lmid; t += T) {
        double w;
        sm.tab_fm[t] = gray_entry(pl, pl.nin, pl.nmid, pl.Pmid, t, &w, nullptr, bin_mid);
        sm.tab_wm[t] = w;
    }
}

// Middle digit values at middle index pm (the reflected Gray code decoded directly).
template <class PL>
static __device__ __forceinline__ int middle_digit(const PL& pl, int pm, int q) {
    int par = 0, v = 0;
    for (int i = pl.nmid - 1; i >= q; --i) {
        const int R = pl.R[pl.nin + i];
        const int d = (pm / pl.Pmid[i]) % R;
        v = (par & 1) ? R - 1 - d : d;
        par += v;
    }
    return v;
}

// ---------------------------------------------------------------------------------------- sweep
// Product of the other three threads' totals of a 4-thread lane: all three are gathered with
// independent shuffles (one shuffle latency), then multiplied.
template <int TPL, typename R>
__device__ __forceinline__ void others_product(R xr, R xi, R& yr, R& yi, unsigned gmask) {
    const R ar = __shfl_xor_sync(gmask, xr, 1), ai = __shfl_xor_sync(gmask, xi, 1);
    const R br = __shfl_xor_sync(gmask, xr, 2), bi = __shfl_xor_sync(gmask, xi, 2);
    const R cr = __shfl_xor_sync(gmask, xr, 3), ci = __shfl_xor_sync(gmask, xi, 3);
    const R tr = fma(ar, br, -(ai * bi)), ti = fma(ar, bi, ai * br);
    yr = fma(tr, cr, -(ti * ci));
    yi = fma(tr, ci, ti * cr);
}

// One term: optional rank-1 update of the column sums (brow != null: s += f b), then
// acc_c += w prod_{j != c} s_j over this thread's KH columns.  The product of the other TPL - 1
// threads' columns of the lane enters the suffix chain (exchanged once per term); w enters the
// prefix chain of the lane's first thread.
template <int KH, int TPL, typename R, typename C2>
__device__ __forceinline__ void term(R (&sr)[KH], R (&si)[KH], R (&ar)[KH], R (&ai)[KH], const C2* brow, R f, R w,
                                     int h, unsigned gmask) {
    R pr[KH], pi[KH];
    if (brow) {
#pragma unroll
        for (int c = 0; c < KH; ++c) {
            const C2 b = brow[c];
            sr[c] = fma(f, (R)b.x, sr[c]);
            si[c] = fma(f, (R)b.y, si[c]);
        }
    }
    const R w0 = (h == 0) ? w : R(1);
    pr[0] = w0;
    pi[0] = R(0);
    R xr = w0 * sr[0], xi = w0 * si[0];
#pragma unroll
    for (int c = 1; c < KH; ++c) {
        pr[c] = xr;
        pi[c] = xi;
        const R nr = fma(xr, sr[c], -(xi * si[c]));
        xi = fma(xr, si[c], xi * sr[c]);
        xr = nr;
    }
    R yr, yi;
    if constexpr (TPL == 1) {
        yr = R(1); yi = R(0);
    } else if constexpr (TPL == 2) {
        yr = __shfl_xor_sync(gmask, xr, 1);
        yi = __shfl_xor_sync(gmask, xi, 1);
    } else {
        others_product<TPL>(xr, xi, yr, yi, gmask);
    }
#pragma unroll
    for (int c = KH - 1; c >= 1; --c) {
        ar[c] = fma(pr[c], yr, ar[c]);
        ar[c] = fma(-pi[c], yi, ar[c]);
        ai[c] = fma(pr[c], yi, ai[c]);
        ai[c] = fma(pi[c], yr, ai[c]);
        const R nr = fma(yr, sr[c], -(yi * si[c]));
        yi = fma(yr, si[c], yi * sr[c]);
        yr = nr;
    }
    ar[0] = fma(pr[0], yr, ar[0]);
    ai[0] = fma(pr[0], yi, ai[0]);
}

// One term with this thread's KH columns split into two halves A = [0, KA) and B = [KA, KH) whose
// product chains run interleaved (two independent dependency chains instead of one).  The half
// totals are folded into the other half's suffix start, so for TPL == 1 this costs no extra
// multiplication; for TPL == 2 the lane total, and the two suffix starts, cost three.
template <int KH, int TPL, typename R, typename C2>
__device__ __forceinline__ void term_split(R (&sr)[KH], R (&si)[KH], R (&ar)[KH], R (&ai)[KH], const C2* brow, R f,
                                           R w, int h, unsigned gmask) {
    constexpr int KA = KH / 2;
    R pr[KH], pi[KH];
    if (brow) {
#pragma unroll
        for (int c = 0; c < KH; ++c) {
            const C2 b = brow[c];
            sr[c] = fma(f, (R)b.x, sr[c]);
            si[c] = fma(f, (R)b.y, si[c]);
        }
    }
    const R w0 = (h == 0) ? w : R(1);
    pr[0] = w0; pi[0] = R(0);
    pr[KA] = R(1); pi[KA] = R(0);
    R xar = w0 * sr[0], xai = w0 * si[0];
    R xbr = sr[KA], xbi = si[KA];
#pragma unroll
    for (int i = 1; i < KH - KA; ++i) {
        if (i < KA) {
            const int c = i;
            pr[c] = xar; pi[c] = xai;
            const R nr = fma(xar, sr[c], -(xai * si[c]));
            xai = fma(xar, si[c], xai * sr[c]);
            xar = nr;
        }
        {
            const int c = KA + i;
            pr[c] = xbr; pi[c] = xbi;
            const R nr = fma(xbr, sr[c], -(xbi * si[c]));
            xbi = fma(xbr, si[c], xbi * sr[c]);
            xbr = nr;
        }
    }
    R yar, yai, ybr, ybi;                 // suffix starts: other half's total times the other threads'
    if constexpr (TPL == 1) {
        yar = xbr; yai = xbi;
        ybr = xar; ybi = xai;
    } else {
        const R tr = fma(xar, xbr, -(xai * xbi)), ti = fma(xar, xbi, xai * xbr);
        const R Yr = __shfl_xor_sync(gmask, tr, 1), Yi = __shfl_xor_sync(gmask, ti, 1);
        yar = fma(xbr, Yr, -(xbi * Yi)); yai = fma(xbr, Yi, xbi * Yr);
        ybr = fma(xar, Yr, -(xai * Yi)); ybi = fma(xar, Yi, xai * Yr);
    }
#pragma unroll
    for (int i = KH - KA - 1; i >= 1; --i) {
        {
            const int c = KA + i;
            ar[c] = fma(pr[c], ybr, ar[c]);
            ar[c] = fma(-pi[c], ybi, ar[c]);
            ai[c] = fma(pr[c], ybi, ai[c]);
            ai[c] = fma(pi[c], ybr, ai[c]);
            const R nr = fma(ybr, sr[c], -(ybi * si[c]));
            ybi = fma(ybr, si[c], ybi * sr[c]);
            ybr = nr;
        }
        if (i < KA) {
            const int c = i;
            ar[c] = fma(pr[c], yar, ar[c]);
            ar[c] = fma(-pi[c], yai, ar[c]);
            ai[c] = fma(pr[c], yai, ai[c]);
            ai[c] = fma(pi[c], yar, ai[c]);
            const R nr = fma(yar, sr[c], -(yai * si[c]));
            yai = fma(yar, si[c], yai * sr[c]);
            yar = nr;
        }
    }
    ar[KA] = fma(pr[KA], ybr, ar[KA]);
    ai[KA] = fma(pr[KA], ybi, ai[KA]);
    ar[0] = fma(pr[0], yar, ar[0]);
    ai[0] = fma(pr[0], yai, ai[0]);
}

// Term dispatch: split chains for wide per-thread column sets of 1- or 2-thread lanes.
template <int KH, int TPL, typename R, typename C2>
__device__ __forceinline__ void term_any(R (&sr)[KH], R (&si)[KH], R (&ar)[KH], R (&ai)[KH], const C2* brow, R f, R w,
                                         int h, unsigned gmask) {
    if constexpr (PE_SPLIT && sizeof(R) == 8 && TPL <= 2 && KH >= 6)
        term_split<KH, TPL, R, C2>(sr, si, ar, ai, brow, f, w, h, gmask);
    else term<KH, TPL, R, C2>(sr, si, ar, ai, brow, f, w, h, gmask);
}

// Two consecutive terms, interleaved for instruction-level parallelism: the first applies the
// update (fa, ba) to s, the second (fb, bb) on top of it; their product chains are independent.
template <int KH, int TPL, typename R, typename C2>
__device__ __forceinline__ void term2(R (&sr)[KH], R (&si)[KH], R (&ar)[KH], R (&ai)[KH], const C2* ba, R fa, R wa,
                                      const C2* bb, R fb, R wb, int h, unsigned gmask) {
    R tr[KH], ti[KH];
#pragma unroll
    for (int c = 0; c < KH; ++c) {
        const C2 x = ba[c], y = bb[c];
        sr[c] = fma(fa, (R)x.x, sr[c]);
        si[c] = fma(fa, (R)x.y, si[c]);
        tr[c] = fma(fb, (R)y.x, sr[c]);
        ti[c] = fma(fb, (R)y.y, si[c]);
    }
    R par[KH], pai[KH], pbr[KH], pbi[KH];
    const R wa0 = (h == 0) ? wa : R(1), wb0 = (h == 0) ? wb : R(1);
    par[0] = wa0; pai[0] = R(0);
    pbr[0] = wb0; pbi[0] = R(0);
    R xar = wa0 * sr[0], xai = wa0 * si[0];
    R xbr = wb0 * tr[0], xbi = wb0 * ti[0];
#pragma unroll
    for (int c = 1; c < KH; ++c) {
        par[c] = xar; pai[c] = xai;
        pbr[c] = xbr; pbi[c] = xbi;
        const R nar = fma(xar, sr[c], -(xai * si[c]));
        xai = fma(xar, si[c], xai * sr[c]);
        xar = nar;
        const R nbr = fma(xbr, tr[c], -(xbi * ti[c]));
        xbi = fma(xbr, ti[c], xbi * tr[c]);
        xbr = nbr;
    }
    R yar, yai, ybr, ybi;
    if constexpr (TPL == 1) {
        yar = R(1); yai = R(0); ybr = R(1); ybi = R(0);
    } else if constexpr (TPL == 2) {
        yar = __shfl_xor_sync(gmask, xar, 1);
        yai = __shfl_xor_sync(gmask, xai, 1);
        ybr = __shfl_xor_sync(gmask, xbr, 1);
        ybi = __shfl_xor_sync(gmask, xbi, 1);
    } else {
        others_product<TPL>(xar, xai, yar, yai, gmask);
        others_product<TPL>(xbr, xbi, ybr, ybi, gmask);
    }
#pragma unroll
    for (int c = KH - 1; c >= 1; --c) {
        ar[c] = fma(par[c], yar, ar[c]);
        ar[c] = fma(-pai[c], yai, ar[c]);
        ai[c] = fma(par[c], yai, ai[c]);
        ai[c] = fma(pai[c], yar, ai[c]);
        ar[c] = fma(pbr[c], ybr, ar[c]);
        ar[c] = fma(-pbi[c], ybi, ar[c]);
        ai[c] = fma(pbr[c], ybi, ai[c]);
        ai[c] = fma(pbi[c], ybr, ai[c]);
        const R nar = fma(yar, sr[c], -(yai * si[c]));
        yai = fma(yar, si[c], yai * sr[c]);
        yar = nar;
        const R nbr = fma(ybr, tr[c], -(ybi * ti[c]));
        ybi = fma(ybr, ti[c], ybi * tr[c]);
        ybr = nbr;
    }
    ar[0] = fma(par[0], yar, ar[0]);
    ai[0] = fma(par[0], yai, ai[0]);
    ar[0] = fma(pbr[0], ybr, ar[0]);
    ai[0] = fma(pbr[0], ybi, ai[0]);
#pragma unroll
    for (int c = 0; c < KH; ++c) { sr[c] = tr[c]; si[c] = ti[c]; }
}

// Walk one inner block forward (fwd) or backward from the current column sums.  `f2` is the
// magnitude of the column-sum step (2 for B, 1 for the pre-doubled B32); w_t = wscale * tab[t].
template <int KH, int TPL, int UNR, typename R, typename C2, typename TabW, class SM, class BMat>
__device__ __forceinline__ void inner_block(R (&sr)[KH], R (&si)[KH], R (&ar)[KH], R (&ai)[KH], const SM& sm,
                                           const BMat& Bm, const TabW* tab, R wscale, R f2, bool fwd, int Lin,
                                           int c0, int h, unsigned gmask) {
    if (fwd) {
        term_any<KH, TPL, R, C2>(sr, si, ar, ai, nullptr, R(0), wscale * (R)tab[0], h, gmask);
        int t = 1;
        if constexpr (UNR == 2) {
            for (; t + 1 < Lin; t += 2) {
                const unsigned ea = sm.tab_f[t], eb = sm.tab_f[t + 1];
                term2<KH, TPL, R, C2>(sr, si, ar, ai, &Bm[ea & 63u][c0], (ea & 0x80u) ? -f2 : f2, wscale * (R)tab[t],
                                      &Bm[eb & 63u][c0], (eb & 0x80u) ? -f2 : f2, wscale * (R)tab[t + 1], h, gmask);
            }
        }
        for (; t < Lin; ++t) {
            const unsigned e = sm.tab_f[t];
            term_any<KH, TPL, R, C2>(sr, si, ar, ai, &Bm[e & 63u][c0], (e & 0x80u) ? -f2 : f2, wscale * (R)tab[t], h, gmask);
        }
    } else {
        term_any<KH, TPL, R, C2>(sr, si, ar, ai, nullptr, R(0), wscale * (R)tab[Lin - 1], h, gmask);
        int t = Lin - 2;
        if constexpr (UNR == 2) {
            for (; t - 1 >= 0; t -= 2) {
                const unsigned ea = sm.tab_f[t + 1], eb = sm.tab_f[t];
                term2<KH, TPL, R, C2>(sr, si, ar, ai, &Bm[ea & 63u][c0], (ea & 0x80u) ? f2 : -f2, wscale * (R)tab[t],
                                      &Bm[eb & 63u][c0], (eb & 0x80u) ? f2 : -f2, wscale * (R)tab[t - 1], h, gmask);
            }
        }
        for (; t >= 0; --t) {
            const unsigned e = sm.tab_f[t + 1];
            term_any<KH, TPL, R, C2>(sr, si, ar, ai, &Bm[e & 63u][c0], (e & 0x80u) ? f2 : -f2, wscale * (R)tab[t], h, gmask);
        }
    }
}

// ---------------------------------------------------------------------------------------- paired FP32
// The mixed form's term on Blackwell's paired FP32 instructions (FFMA2 / FMUL2: two lanes of a float2 in
// one issue slot).  A thread's KH columns are two halves [0, KA) and [KA, KH) whose product chains run
// side by side in the two halves of every float2: sr[c] = (re s_c, re s_{KA+c}), si[c] likewise, and the
// same for the prefix products and the accumulators.  Arithmetic as term_split (FP32).
static __device__ __forceinline__ float2 f2neg(float2 a) { return make_float2(-a.x, -a.y); }

template <int KH, int TPL>
__device__ __forceinline__ void term_pair(float2 (&sr)[KH / 2], float2 (&si)[KH / 2], float2 (&ar)[KH / 2],
                                          float2 (&ai)[KH / 2], const float4* brow, float f, float w, int h,
                                          unsigned gmask) {
    constexpr int KA = KH / 2;
    if (brow) {
        const float2 ff = make_float2(f, f);
#pragma unroll
        for (int c = 0; c < KA; ++c) {
            const float4 b = brow[c];
            sr[c] = __ffma2_rn(ff, make_float2(b.x, b.y), sr[c]);
            si[c] = __ffma2_rn(ff, make_float2(b.z, b.w), si[c]);
        }
    }
    const float2 w0 = make_float2((h == 0) ? w : 1.0f, 1.0f);
    float2 pr[KA], pi[KA];
    pr[0] = w0;
    pi[0] = make_float2(0.0f, 0.0f);
    float2 xr = __fmul2_rn(w0, sr[0]), xi = __fmul2_rn(w0, si[0]);
#pragma unroll
    for (int c = 1; c < KA; ++c) {
        pr[c] = xr;
        pi[c] = xi;
        const float2 nr = __ffma2_rn(xr, sr[c], f2neg(__fmul2_rn(xi, si[c])));
        xi = __ffma2_rn(xr, si[c], __fmul2_rn(xi, sr[c]));
        xr = nr;
    }
    float2 yr, yi;                        // suffix starts: (other half's total) x (the partner's total)
    if constexpr (TPL == 1) {
        yr = make_float2(xr.y, xr.x);
        yi = make_float2(xi.y, xi.x);
    } else {
        const float tr = fmaf(xr.x, xr.y, -(xi.x * xi.y)), ti = fmaf(xr.x, xi.y, xi.x * xr.y);
        const float Yr = __shfl_xor_sync(gmask, tr, 1), Yi = __shfl_xor_sync(gmask, ti, 1);
        const float2 br = make_float2(xr.y, xr.x), bi = make_float2(xi.y, xi.x);
        const float2 YR = make_float2(Yr, Yr), YI = make_float2(Yi, Yi);
        yr = __ffma2_rn(br, YR, f2neg(__fmul2_rn(bi, YI)));
        yi = __ffma2_rn(br, YI, __fmul2_rn(bi, YR));
    }
#pragma unroll
    for (int c = KA - 1; c >= 1; --c) {
        ar[c] = __ffma2_rn(pr[c], yr, ar[c]);
        ar[c] = __ffma2_rn(f2neg(pi[c]), yi, ar[c]);
        ai[c] = __ffma2_rn(pr[c], yi, ai[c]);
        ai[c] = __ffma2_rn(pi[c], yr, ai[c]);
        const float2 nr = __ffma2_rn(yr, sr[c], f2neg(__fmul2_rn(yi, si[c])));
        yi = __ffma2_rn(yr, si[c], __fmul2_rn(yi, sr[c]));
        yr = nr;
    }
    ar[0] = __ffma2_rn(pr[0], yr, ar[0]);
    ai[0] = __ffma2_rn(pr[0], yi, ai[0]);
}

// One paired inner block, forward or backward (B32 pre-doubled: the update magnitude is 1).
template <int KH, int TPL, class SM>
__device__ __forceinline__ void inner_block_pair(float2 (&sr)[KH / 2], float2 (&si)[KH / 2], float2 (&ar)[KH / 2],
                                                 float2 (&ai)[KH / 2], const SM& sm, bool fwd, int Lin, int h,
                                                 unsigned gmask) {
    constexpr int KA = KH / 2;
    const int q0 = h * KA;
    if (fwd) {
        term_pair<KH, TPL>(sr, si, ar, ai, nullptr, 0.0f, sm.tab_w32[0], h, gmask);
        for (int t = 1; t < Lin; ++t) {
            const unsigned e = sm.tab_f[t];
            term_pair<KH, TPL>(sr, si, ar, ai, reinterpret_cast<const float4*>(&sm.B32[e & 63u][0]) + q0,
                               (e & 0x80u) ? -1.0f : 1.0f, sm.tab_w32[t], h, gmask);
        }
    } else {
        term_pair<KH, TPL>(sr, si, ar, ai, nullptr, 0.0f, sm.tab_w32[Lin - 1], h, gmask);
        for (int t = Lin - 2; t >= 0; --t) {
            const unsigned e = sm.tab_f[t + 1];
            term_pair<KH, TPL>(sr, si, ar, ai, reinterpret_cast<const float4*>(&sm.B32[e & 63u][0]) + q0,
                               (e & 0x80u) ? 1.0f : -1.0f, sm.tab_w32[t], h, gmask);
        }
    }
}

// Deterministic reduction of the per-thread accumulators over the lanes of the CTA -> sm.P.
template <int KH, int TPL, class SM>
__device__ __forceinline__ void reduce_to_P(double (&ar)[KH], double (&ai)[KH], SM& sm, int c0) {
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

// High-digit values of Gray lane hl (plain mixed radix over the high digits), packed HBITS bits per
// digit for the first HDIG digits (5 x 12 when radices are <= 32, 6 x 10 for the wide tiers), and the
// lane's weight prod (-1)^v C(M, v) over them.
template <class PL>
struct HighPack {
    static constexpr int HBITS = PL::NKMAX <= NARROW ? 5 : 6;
    static constexpr int HDIG = 60 / HBITS;
};
template <class PL>
static __device__ __forceinline__ uint64_t lane_digits(const PL& pl, int64_t hl, double* wh_out) {
    const int hi0 = pl.nin + pl.nmid;
    uint64_t packed = 0;
    double wh = 1.0;
    int64_t rem = hl;
    for (int i = 0; i < pl.nhi; ++i) {
        const int R = pl.R[hi0 + i];
        int v;
        if (R == 2) { v = (int)(rem & 1); rem >>= 1; }      // the common radix without a 64-bit division
        else { v = (int)(rem % R); rem /= R; }
        if (i < HighPack<PL>::HDIG) packed |= (uint64_t)v << (HighPack<PL>::HBITS * i);
        wh *= signed_binom(pl.M[hi0 + i], v);
    }
    *wh_out = wh;
    return packed;
}

// Column sums of one lane at a given digit state, FP64: s_j = sum_kd (M_kd - 2 v_kd) B[kd][j] with the
// inner digits at their start (0) or end (vend) state, the middle digits at middle index pm and the
// high digits of the lane (packed by lane_digits; more than 12 high digits are decoded from hl).
template <int KH, class SM>
__device__ __forceinline__ void lane_sums(const SM& sm, int c0, bool inner_end, int pm, int64_t hl, uint64_t hpack,
                                          double (&xr)[KH], double (&xi)[KH]) {
    const auto& pl = sm.plan;
    using HP = HighPack<decltype(sm.plan)>;
#pragma unroll
    for (int j = 0; j < KH; ++j) { xr[j] = 0.0; xi[j] = 0.0; }
    const int nin = pl.nin, nmid = pl.nmid, hi0 = nin + nmid, nhi = pl.nhi;
    auto add = [&](int kd, int v) {
        const double c = (double)(pl.M[kd] - 2 * v);
        const double2* b = &sm.B[kd][c0];
#pragma unroll
        for (int j = 0; j < KH; ++j) { xr[j] = fma(c, b[j].x, xr[j]); xi[j] = fma(c, b[j].y, xi[j]); }
    };
    for (int kd = 0; kd < nin; ++kd) add(kd, inner_end ? sm.plan.vend[kd] : 0);
    int par = 0;                                       // middle digits top-down (reflected Gray)
    for (int q = nmid - 1; q >= 0; --q) {
        const int R = pl.R[nin + q];
        const int d = (pm / pl.Pmid[q]) % R;
        const int v = (par & 1) ? R - 1 - d : d;
        par += v;
        add(nin + q, v);
    }
    int64_t rem = hl;
    for (int i = 0; i < nhi; ++i) {
        int v;
        if (i < HP::HDIG) {
            v = (int)((hpack >> (HP::HBITS * i)) & ((1u << HP::HBITS) - 1u));
        } else {
            int64_t r2 = hl;
            for (int q = 0; q < i; ++q) r2 /= pl.R[hi0 + q];
            v = (int)(r2 % pl.R[hi0 + i]);
        }
        add(hi0 + i, v);
    }
    (void)rem;
    for (int kd = hi0 + nhi; kd < pl.D; ++kd) add(kd, 0);
}

// FP64 sweep of tier KP (columns padded to KP: padded column sums hold 1, their B rows are zero).
template <int KP, int TPL, class SM>
__device__ void sweep_f64(SM& sm) {
    constexpr int KH = KP / TPL;
    const auto& pl = sm.plan;
    const int tid = threadIdx.x;
    const int lanes = blockDim.x / TPL, lane = tid / TPL, h = tid % TPL, c0 = h * KH;
    const int wl0 = (tid & ~31) / TPL;                     // first lane of this warp
    const unsigned gmask = 0xffffffffu;                    // the warp walks its lanes in lockstep
    const int K = pl.K, Lin = pl.Lin, Lmid = pl.Lmid, nin = pl.nin;
    const int64_t H = pl.H;
    double ar[KH], ai[KH];
#pragma unroll
    for (int j = 0; j < KH; ++j) { ar[j] = 0.0; ai[j] = 0.0; }
    for (int64_t hw = sm.lane0 + wl0; hw < H; hw += (int64_t)lanes * sm.lane_mult) {
        double sr[KH], si[KH], wh;
        int64_t hl = hw + (lane - wl0);
        const bool live = hl < H;                          // a lane past the end repeats lane H - 1 at weight 0
        if (!live) hl = H - 1;
        const uint64_t hpack = lane_digits(pl, hl, &wh);
        if (!live) wh = 0.0;
        lane_sums<KH>(sm, c0, false, 0, hl, hpack, sr, si);
#pragma unroll
        for (int j = 0; j < KH; ++j) if (c0 + j >= K) { sr[j] = 1.0; si[j] = 0.0; }
        for (int pm = 0; pm < Lmid; ++pm) {
            if (pm > 0) {
                const unsigned e = sm.tab_fm[pm];
                const double f = (e & 0x80u) ? -2.0 : 2.0;
                const double2* b = &sm.B[nin + (e & 63u)][c0];
#pragma unroll
                for (int j = 0; j < KH; ++j) { sr[j] = fma(f, b[j].x, sr[j]); si[j] = fma(f, b[j].y, si[j]); }
            }
            const double wmh = wh * sm.tab_wm[pm];
            inner_block<KH, TPL, PE_UNROLL, double, double2, double>(sr, si, ar, ai, sm, sm.B, sm.tab_w, wmh, 2.0,
                                                                    !(pm & 1), Lin, c0, h, gmask);
        }
    }
    reduce_to_P<KH, TPL>(ar, ai, sm, c0);
}

// Mixed sweep: every inner block starts from column sums formed in FP64 from the digit values
// (no drift carried across blocks), runs in complex FP32, and is folded into FP64 accumulators.
template <int KP, int TPL, class SM>
__device__ void sweep_mixed(SM& sm) {
    constexpr int KH = KP / TPL;
    const auto& pl = sm.plan;
    const int tid = threadIdx.x;
    const int lanes = blockDim.x / TPL, lane = tid / TPL, h = tid % TPL, c0 = h * KH;
    const int wl0 = (tid & ~31) / TPL;
    const unsigned gmask = 0xffffffffu;
    const int K = pl.K, Lin = pl.Lin, Lmid = pl.Lmid;
    const int64_t H = pl.H;
    double ar[KH], ai[KH];
#pragma unroll
    for (int j = 0; j < KH; ++j) { ar[j] = 0.0; ai[j] = 0.0; }
    for (int64_t hw = sm.lane0 + wl0; hw < H; hw += (int64_t)lanes * sm.lane_mult) {
        double wh;
        int64_t hl = hw + (lane - wl0);
        const bool live = hl < H;
        if (!live) hl = H - 1;
        const uint64_t hpack = lane_digits(pl, hl, &wh);
        if (!live) wh = 0.0;
        for (int pm = 0; pm < Lmid; ++pm) {
            const bool fwd = !(pm & 1);
            float sr[KH], si[KH];
            {
                double xr[KH], xi[KH];
                lane_sums<KH>(sm, c0, !fwd, pm, hl, hpack, xr, xi);
#pragma unroll
                for (int j = 0; j < KH; ++j) {
                    const bool pad = c0 + j >= K;
                    sr[j] = pad ? 1.0f : (float)xr[j];
                    si[j] = pad ? 0.0f : (float)xi[j];
                }
            }
            const double wmh = wh * sm.tab_wm[pm];
            if constexpr (PE_PAIR32 && TPL <= 2 && KH % 2 == 0) {
                constexpr int KA = KH / 2;
                float2 s2r[KA], s2i[KA], a2r[KA], a2i[KA];
#pragma unroll
                for (int c = 0; c < KA; ++c) {
                    s2r[c] = make_float2(sr[c], sr[KA + c]);
                    s2i[c] = make_float2(si[c], si[KA + c]);
                    a2r[c] = make_float2(0.0f, 0.0f);
                    a2i[c] = make_float2(0.0f, 0.0f);
                }
                inner_block_pair<KH, TPL>(s2r, s2i, a2r, a2i, sm, fwd, Lin, h, gmask);
#pragma unroll
                for (int c = 0; c < KA; ++c) {
                    ar[c] = fma(wmh, (double)a2r[c].x, ar[c]);
                    ai[c] = fma(wmh, (double)a2i[c].x, ai[c]);
                    ar[KA + c] = fma(wmh, (double)a2r[c].y, ar[KA + c]);
                    ai[KA + c] = fma(wmh, (double)a2i[c].y, ai[KA + c]);
                }
            } else {
                float a32r[KH], a32i[KH];
#pragma unroll
                for (int j = 0; j < KH; ++j) { a32r[j] = 0.0f; a32i[j] = 0.0f; }
                inner_block<KH, TPL, PE_UNROLL, float, float2, float>(sr, si, a32r, a32i, sm, sm.B32, sm.tab_w32, 1.0f,
                                                                     1.0f, fwd, Lin, c0, h, gmask);
#pragma unroll
                for (int j = 0; j < KH; ++j) {
                    ar[j] = fma(wmh, (double)a32r[j], ar[j]);
                    ai[j] = fma(wmh, (double)a32i[j], ai[j]);
                }
            }
        }
    }
    reduce_to_P<KH, TPL>(ar, ai, sm, c0);
}

#define PE_TIER(KPv, CALL)                                   \
    if constexpr (KPM >= KPv) {                              \
        if (K <= KPv) { CALL; return; }                      \
    }

template <int TPL, int KPM, class SM>
__device__ void dispatch_f64(SM& sm, int K) {
    PE_TIER(4, (sweep_f64<4, TPL>(sm)))
    PE_TIER(8, (sweep_f64<8, TPL>(sm)))
    PE_TIER(12, (sweep_f64<12, TPL>(sm)))
    PE_TIER(16, (sweep_f64<16, TPL>(sm)))
    PE_TIER(20, (sweep_f64<20, TPL>(sm)))
    PE_TIER(24, (sweep_f64<24, TPL>(sm)))
    PE_TIER(28, (sweep_f64<28, TPL>(sm)))
    PE_TIER(32, (sweep_f64<32, TPL>(sm)))
    PE_TIER(36, (sweep_f64<36, TPL>(sm)))
    PE_TIER(40, (sweep_f64<40, TPL>(sm)))
    PE_TIER(44, (sweep_f64<44, TPL>(sm)))
    PE_TIER(48, (sweep_f64<48, TPL>(sm)))
    PE_TIER(52, (sweep_f64<52, TPL>(sm)))
    PE_TIER(56, (sweep_f64<56, TPL>(sm)))
    PE_TIER(60, (sweep_f64<60, TPL>(sm)))
    PE_TIER(64, (sweep_f64<64, TPL>(sm)))
}

template <int TPL, int KPM, class SM>
__device__ void dispatch_mixed(SM& sm, int K) {
    PE_TIER(4, (sweep_mixed<4, TPL>(sm)))
    PE_TIER(8, (sweep_mixed<8, TPL>(sm)))
    PE_TIER(12, (sweep_mixed<12, TPL>(sm)))
    PE_TIER(16, (sweep_mixed<16, TPL>(sm)))
    PE_TIER(20, (sweep_mixed<20, TPL>(sm)))
    PE_TIER(24, (sweep_mixed<24, TPL>(sm)))
    PE_TIER(28, (sweep_mixed<28, TPL>(sm)))
    PE_TIER(32, (sweep_mixed<32, TPL>(sm)))
}
}  // namespace pe

#include "fock_comp.cuh"

namespace pe {

// One cofactor step of the stream held in shared memory (K1 >= 1): plan, prepare, sweep.  PREC: 0 FP64,
// 1 mixed, 2 compensated mixed.
template <int TPL, int KPM, int PREC, class SM>
__device__ __forceinline__ void cofactor_step(SM& sm, const double2* A, int64_t rs, int64_t cs, int K1, int K) {
    constexpr bool MIXED = PREC == PREC_MIXED;
    if (threadIdx.x < 32) plan_step(sm, K1, K, blockDim.x / TPL * sm.lane_mult, MIXED ? MIXED_LIN : LIN_MAX, MID_MAX);
    __syncthreads();
    // paired FP32 sweeps (mixed form, 1- and 2-thread lanes): columns per thread of the dispatched tier
    const int kh = (MIXED && PE_PAIR32 && TPL <= 2) ? ((K + 3) / 4 * 4) / TPL : 0;
    prepare_step(sm, A, rs, cs, MIXED, kh);
    __syncthreads();
    if constexpr (PREC == PREC_COMP) {
        prepare_comp(sm, ((K + 3) / 4 * 4) / TPL, TPL);
        __syncthreads();
        dispatch_comp<TPL, KPM>(sm, K);
    } else if constexpr (MIXED) {
        dispatch_mixed<TPL, KPM>(sm, K);
    } else {
        dispatch_f64<TPL, KPM>(sm, K);
    }
}

// ---------------------------------------------------------------------------------------- draw
// Marginal over the m output modes, FP64 block scan (contiguous chunk per thread, warp scan, warps
// in order), then idx = min(#{rho : cw_rho < u * tot}, m - 1) with tot = cw[m - 1]
// (cofactors_triton.py:298-308).  Thread 0 records the pick and updates the groups; the gap
// min |cw - u tot| / tot is left in sm.fmin[0].
template <class SM>
static __device__ void draw_step(SM& sm, double* __restrict__ wgt, const double2* __restrict__ A, int64_t rs, int64_t cs,
                                 int m, int k, double u, double* __restrict__ marg_row, bool update_groups) {
    const int tid = threadIdx.x, T = blockDim.x, lid = tid & 31, wid = tid >> 5, nw = T >> 5;
    // DR modes per thread at a time, and the column loop unrolled 4 times, so that 16 independent loads of
    // A (from L2) are in flight instead of one; the sum over columns keeps its order (same bits as one mode
    // at a time).  The draw is bound by L2 latency, not by its few FLOPs (m = 900, the c3 batch: 4-5 %
    // faster than two columns ahead).
    constexpr int DR = 4;
    for (int rho0 = tid; rho0 < m; rho0 += T * DR) {
        double xr[DR], xi[DR];
#pragma unroll
        for (int r = 0; r < DR; ++r) { xr[r] = 0.0; xi[r] = 0.0; }
#pragma unroll 4
        for (int c = 0; c < k; ++c) {
            const int64_t co = (int64_t)sm.cols[c] * cs;
            const double2 p = sm.P[c];
            double2 a[DR];
#pragma unroll
            for (int r = 0; r < DR; ++r) {
                const int rho = rho0 + r * T;
                a[r] = rho < m ? A[(int64_t)rho * rs + co] : make_double2(0.0, 0.0);
            }
#pragma unroll
            for (int r = 0; r < DR; ++r) {
                xr[r] = fma(a[r].x, p.x, xr[r]);
                xr[r] = fma(-a[r].y, p.y, xr[r]);
                xi[r] = fma(a[r].x, p.y, xi[r]);
                xi[r] = fma(a[r].y, p.x, xi[r]);
            }
        }
#pragma unroll
        for (int r = 0; r < DR; ++r) {
            const int rho = rho0 + r * T;
            if (rho < m) wgt[rho] = xr[r] * xr[r] + xi[r] * xi[r];
        }
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
        const int pick = min(c, m - 1);
        sm.rows[k - 1] = pick;
        sm.fmin[0] = g / tot;
        if (update_groups) add_to_groups(sm, pick);
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------------------- chain
template <int TPL, int KPM, int PREC>
__device__ void chain_one(const ChainParams& p, SmemFor<KPM, PREC>& sm, double* wgt, int64_t s, bool stop_early) {
    const int tid = threadIdx.x;
    const int64_t g = p.dp[s];
    bool ok = g >= 0 && g < p.G;
    int m = 0, nin = 0;
    int64_t off = 0;
    if (ok) { m = p.inst_m[g]; nin = p.inst_n[g]; off = p.inst_off[g]; }
    const int nk = p.nk ? p.nk[s] : p.n_stride;
    const int kf = p.k_first;
    if (nk < kf - 1) return;                                  // nothing to run (a dropped stream)
    ok = ok && nk >= 0 && nk <= p.n_stride && nk <= KPM && m >= 1 && m <= p.m_cap && m <= p.occ_stride;
    if (ok && tid < nk) {
        const int64_t c = p.cols[s * p.n_stride + tid];
        if (c < 0 || c >= nin) atomicOr(&sm.bad, 1);
        else sm.cols[tid] = (int)c;
    }
    if (ok && tid < kf - 1) {
        const int64_t r = p.rows[s * p.n_stride + tid];
        if (r < 0 || r >= m) atomicOr(&sm.bad, 1);
        else sm.rows[tid] = (int)r;
    }
    if (!ok && tid == 0) sm.bad = 1;
    if (tid == 0) { sm.ngrp = 0; sm.lane0 = 0; sm.lane_mult = 1; }
    __syncthreads();
    if (sm.bad) {
        if (tid == 0) record_error(p.status, p.detail, s);
        return;
    }
    if (kf > 1) {
        if (tid < 32) build_groups_warp(sm, kf - 1);
        __syncthreads();
    }
    const double2* A = p.acol + off;      // (rho, j) at A[j * m + rho]
    const int kend = (stop_early && p.k_stop > 0 && p.k_stop < nk) ? p.k_stop : nk;
    for (int k = kf; k <= kend; ++k) {
        const int K = k, K1 = k - 1;
        if (K1 == 0) {
            if (tid == 0) sm.P[0] = make_double2(1.0, 0.0);
            __syncthreads();
        } else {
            cofactor_step<TPL, KPM, PREC>(sm, A, 1, m, K1, K);
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
        if constexpr (PREC != PREC_F64) {
            draw_step(sm, wgt, A, 1, m, m, k, u, mrow, false);
            if (K1 > 0 && sm.fmin[0] <= guard_band(p, k)) {   // uniform: read after the draw's final barrier
                dispatch_f64<4, KPM>(sm, K);
                draw_step(sm, wgt, A, 1, m, m, k, u, mrow, false);
            }
            if (tid == 0) add_to_groups(sm, sm.rows[k - 1]);
            __syncthreads();
        } else {
            draw_step(sm, wgt, A, 1, m, m, k, u, mrow, true);
        }
    }
    for (int j = kf - 1 + tid; j < kend; j += blockDim.x) p.rows[s * p.n_stride + j] = sm.rows[j];
    if (p.occ && kend == nk) {
        for (int rho = tid; rho < p.occ_stride; rho += blockDim.x) {
            int c = 0;
            for (int j = 0; j < nk; ++j) c += (sm.rows[j] == rho) ? 1 : 0;
            p.occ[s * (int64_t)p.occ_stride + rho] = c;
        }
    }
}


template <int TPL, int KPM, int PREC>
__global__ void __launch_bounds__(PE_MAXT, PE_MINB) fock_chain_kernel(ChainParams p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using SM = SmemFor<KPM, PREC>;
    SM& sm = *reinterpret_cast<SM*>(smem_raw);
    double* wgt = reinterpret_cast<double*>(smem_raw + smem_fixed_bytes<KPM, PREC>());
    const int tid = threadIdx.x;
    for (;;) {
        if (tid == 0) {
            const unsigned long long q = atomicAdd(p.queue, 1ull);
            sm.cur = queue_stream(p, q);
            sm.lane0 = (int64_t)q;                  // the ticket, until chain_one resets the field
            sm.bad = 0;
        }
        __syncthreads();
        const int64_t s = sm.cur;
        const bool stop_early = p.split_cap < 0 || sm.lane0 < p.split_cap;
        __syncthreads();
        if (s < 0) return;
        if (s >= p.S) {
            if (tid == 0) record_error(p.status, p.detail, s);
            return;
        }
        chain_one<TPL, KPM, PREC>(p, sm, wgt, s, stop_early);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------- split steps
// A heavy step of few streams spread over several CTAs per stream: `split_partial_kernel` computes, for
// work item (stream s, chunk i), the Gray lanes i*lanes + j*(nch*lanes) of step k into
// partial[s][i][:]; `split_draw_kernel` sums a stream's chunks in a fixed order and draws.  The stream
// state between steps (rows chosen so far) lives in the rows output.
struct SplitParams {
    ChainParams c;
    int k;                  // the step (k columns, k - 1 chosen rows), k >= 2
    int nch;                // CTAs per stream at this step
    int64_t nq;             // slots: streams 0..S-1 (no queue range), or queue positions 0..nq-1 of the range
    double2* partial;       // [nq][nch][MAXN]
    int* flag;              // [nq] mixed forms: 1 when the draw fell in the guard band (redo this step in FP64)
    int pass;               // 0: the step; 1: only the flagged streams (FP64 kernels)
};

// The stream of split slot q: q itself without a queue range; with one, the stream at queue position q of
// the range order[lo .. hi), or -1 past its end (or for an invalid range, which the persistent kernel
// records).  Uniform across the CTA.
static __device__ __forceinline__ int64_t split_stream(const ChainParams& p, int64_t q) {
    if (!p.qrange) return q;
    const int64_t lo = p.qrange[0], hi = p.qrange[1];
    if (lo < 0 || hi > p.S || lo > hi || lo + q >= hi) return -1;
    return p.order ? p.order[lo + q] : lo + q;
}

// Stream state of step k from global memory into shared memory; false when the stream has fewer photons
// than k (nothing to do) or an index is out of range (recorded).  Uniform across the CTA.
template <class SM>
static __device__ bool load_state(const ChainParams& p, SM& sm, int64_t s, int k, int& m, int64_t& off) {
    const int tid = threadIdx.x;
    if (tid == 0) { sm.bad = 0; sm.ngrp = 0; }
    __syncthreads();
    const int64_t g = p.dp[s];
    bool ok = g >= 0 && g < p.G;
    int nin = 0;
    m = 0;
    off = 0;
    if (ok) { m = p.inst_m[g]; nin = p.inst_n[g]; off = p.inst_off[g]; }
    const int nk = p.nk ? p.nk[s] : p.n_stride;
    if (ok && nk < k) return false;
    ok = ok && nk <= p.n_stride && m >= 1 && m <= p.m_cap && m <= p.occ_stride;
    if (ok && tid < k) {
        const int64_t c = p.cols[s * p.n_stride + tid];
        if (c < 0 || c >= nin) atomicOr(&sm.bad, 1);
        else sm.cols[tid] = (int)c;
    }
    if (ok && tid < k - 1) {
        const int64_t r = p.rows[s * p.n_stride + tid];
        if (r < 0 || r >= m) atomicOr(&sm.bad, 1);
        else sm.rows[tid] = (int)r;
    }
    if (!ok && tid == 0) sm.bad = 1;
    __syncthreads();
    if (sm.bad) {
        if (tid == 0) record_error(p.status, p.detail, s);
        return false;
    }
    if (tid < 32) build_groups_warp(sm, k - 1);
    __syncthreads();
    return true;
}

template <int TPL, int KPM, int PREC>
__global__ void __launch_bounds__(PE_MAXT, PE_MINB) split_partial_kernel(SplitParams sp) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using SM = SmemFor<KPM, PREC>;
    SM& sm = *reinterpret_cast<SM*>(smem_raw);
    const ChainParams& p = sp.c;
    const int tid = threadIdx.x, k = sp.k;
    for (int64_t item = blockIdx.x; item < sp.nq * sp.nch; item += gridDim.x) {
        const int64_t q = item / sp.nch;
        const int i = (int)(item % sp.nch);
        const int64_t s = split_stream(p, q);
        if (s < 0 || s >= p.S) continue;                    // past the range's end: nothing (uniform)
        int m;
        int64_t off;
        const bool live = (sp.pass == 0 || sp.flag[q] != 0) && load_state(p, sm, s, k, m, off);
        if (live) {
            if (tid == 0) { sm.lane0 = (int64_t)i * (blockDim.x / TPL); sm.lane_mult = sp.nch; }
            __syncthreads();
            cofactor_step<TPL, KPM, PREC>(sm, p.acol + off, 1, m, k - 1, k);
            if (tid < k) sp.partial[(q * sp.nch + i) * MAXN + tid] = sm.P[tid];
        }
        __syncthreads();
    }
}

// TPL does not enter the draw; it keeps the kernel's symbol distinct in every variant object, whose
// launch bounds differ (one shared symbol would let the runtime launch any object's copy).
template <int TPL, int KPM, int PREC>
__global__ void __launch_bounds__(PE_MAXT, PE_MINB) split_draw_kernel(SplitParams sp) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using SM = SmemFor<KPM, PREC>;
    SM& sm = *reinterpret_cast<SM*>(smem_raw);
    double* wgt = reinterpret_cast<double*>(smem_raw + smem_fixed_bytes<KPM, PREC>());
    const ChainParams& p = sp.c;
    const int tid = threadIdx.x, k = sp.k;
    for (int64_t q = blockIdx.x; q < sp.nq; q += gridDim.x) {
        const int64_t s = split_stream(p, q);
        if (s < 0 || s >= p.S) continue;                    // past the range's end: nothing (uniform)
        int m;
        int64_t off;
        if ((sp.pass == 1 && sp.flag[q] == 0) || !load_state(p, sm, s, k, m, off)) { __syncthreads(); continue; }
        if (tid < k) {
            double xr = 0.0, xi = 0.0;
#pragma unroll 8
            for (int i = 0; i < sp.nch; ++i) {                 // fixed order; unrolled: loads in flight
                const double2 v = sp.partial[(q * sp.nch + i) * MAXN + tid];
                xr += v.x;
                xi += v.y;
            }
            sm.P[tid] = make_double2(xr, xi);
        }
        __syncthreads();
        const double2* A = p.acol + off;
        double u;
        if (p.uniforms) {
            u = p.uniforms[s * p.n_stride + (k - 1)];
        } else {
            const int64_t row = p.seed_row ? p.seed_row[s] : 0;
            const int64_t ro = p.rng_off ? p.rng_off[s] : s;
            u = chain_uniform((uint64_t)p.seeds[row * p.n_stride + (k - 1)], ro);
        }
        double* mrow = p.marg ? p.marg + ((size_t)s * p.n_stride + (k - 1)) * p.marg_stride : nullptr;
        draw_step(sm, wgt, A, 1, m, m, k, u, mrow, false);
        if constexpr (PREC != PREC_F64) {
            const bool redo = sm.fmin[0] <= guard_band(p, k);   // guard band: the FP64 pass redoes this step
            if (tid == 0) sp.flag[q] = redo ? 1 : 0;
            if (redo) { __syncthreads(); continue; }
        } else {
            if (sp.pass == 1 && tid == 0) sp.flag[q] = 0;
        }
        if (tid == 0) p.rows[s * p.n_stride + (k - 1)] = sm.rows[k - 1];
        const int nk = p.nk ? p.nk[s] : p.n_stride;
        if (p.occ && k == nk) {
            for (int rho = tid; rho < p.occ_stride; rho += blockDim.x) {
                int c = 0;
                for (int j = 0; j < k; ++j) c += (sm.rows[j] == rho) ? 1 : 0;
                p.occ[s * (int64_t)p.occ_stride + rho] = c;
            }
        }
        __syncthreads();
    }
}

// Cofactors of S independent blocks: A [S][m][K] row-major, rows [S][K - 1].
template <int TPL, int KPM, int PREC>
__global__ void __launch_bounds__(256) cofactor_kernel(const double2* __restrict__ A, const int64_t* __restrict__ rows,
                                                       int64_t S, int m, int K, double2* __restrict__ P,
                                                       int* status, long long* detail) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using SM = SmemFor<KPM, PREC>;
    SM& sm = *reinterpret_cast<SM*>(smem_raw);
    const int tid = threadIdx.x;
    for (int64_t s = blockIdx.x; s < S; s += gridDim.x) {
        if (tid == 0) { sm.bad = 0; sm.ngrp = 0; sm.lane0 = 0; sm.lane_mult = 1; }
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
        if (tid < 32) build_groups_warp(sm, K - 1);
        __syncthreads();
        if (K == 1) {
            if (tid == 0) sm.P[0] = make_double2(1.0, 0.0);
            __syncthreads();
        } else {
            cofactor_step<TPL, KPM, PREC>(sm, A + s * (int64_t)m * K, K, 1, K - 1, K);
        }
        if (tid < K) P[s * K + tid] = sm.P[tid];
        __syncthreads();
    }
}

}  // namespace pe
