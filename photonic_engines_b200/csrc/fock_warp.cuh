// Warp-per-stream form of the chain kernel, for short chains (at most 16 photons): every warp of a CTA
// runs its own stream, so the per-step work (plan, schedules, draw) of many streams proceeds at once
// and nothing waits on a CTA-wide barrier.  Same algorithm, plan, Gray schedules, all-but-one products,
// draw rule and uniforms as the CTA form (fock_kernels.cuh); the lanes of the collapsed sum are the
// warp's 32 / TPL thread groups.  Up to 128 modes the marginal's weights stay in registers and one pass
// forms the CDF and the pick; beyond, the CDF is formed in 32-mode chunks twice (once for the total, once
// for the pick) instead of being stored, so any number of modes fits.
#pragma once
#include "fock_kernels.cuh"

namespace pe {

constexpr int WMAXN = 16;      // photons per stream
constexpr int WLIN = 128;      // inner schedule length
constexpr int WMID = 128;      // middle schedule length
constexpr int WARPS = 8;       // warps (streams in flight) per CTA

template <int NK>
struct WarpSmemT {
    static constexpr int NKMAX = NK;
    PlanT<NK> plan;
    double2 P[NK];
    double2 B[NK][NK];
    float2 B32[NK][NK];
    double tab_w[WLIN];
    float tab_w32[WLIN];
    double tab_wm[WMID];
    unsigned char tab_f[WLIN];
    unsigned char tab_fm[WMID];
    int rows[NK];
    int cols[NK];
    int grow[NK];
    int gmul[NK];
    int ngrp;
    int bad;
    int64_t cur;
    int64_t lane0;
    int lane_mult;
};
using WarpSmem = WarpSmemT<WMAXN>;    // the largest slice (streams of up to 16 photons)

// Gather B and fill the schedules, lane-parallel.  Element (rho, j) of the instance is A[rho + j * m].
template <class WS>
static __device__ void prepare_warp(WS& sm, const double2* __restrict__ A, int m, bool mixed) {
    constexpr int NW = WS::NKMAX;
    const auto& pl = sm.plan;
    const int lane = threadIdx.x & 31;
    // the gather from L2 with GB independent loads in flight per lane before any store
    constexpr int GB = 8;
    const int nel = pl.D * NW;
    for (int base = lane; base < nel; base += 32 * GB) {
        double2 v[GB];
#pragma unroll
        for (int g = 0; g < GB; ++g) {
            const int idx = base + 32 * g;
            const bool ok = idx < nel && idx % NW < pl.K;
            const int kd = ok ? idx / NW : 0, j = ok ? idx % NW : 0;     // in range even when not loaded
            v[g] = ok ? A[(int64_t)pl.drow[kd] + (int64_t)sm.cols[j] * m] : make_double2(0.0, 0.0);
        }
#pragma unroll
        for (int g = 0; g < GB; ++g) {
            const int idx = base + 32 * g;
            if (idx < nel) {
                const int kd = idx / NW, j = idx % NW;
                sm.B[kd][j] = v[g];
                if (mixed) sm.B32[kd][j] = make_float2((float)(2.0 * v[g].x), (float)(2.0 * v[g].y));
            }
        }
    }
    bool bin_in = true, bin_mid = true;             // schedules of radix-2 digits only (distinct rows)
    for (int q = 0; q < pl.nin; ++q) bin_in = bin_in && pl.R[q] == 2;
    for (int q = 0; q < pl.nmid; ++q) bin_mid = bin_mid && pl.R[pl.nin + q] == 2;
    for (int t = lane; t < pl.Lin; t += 32) {
        double w;
        sm.tab_f[t] = gray_entry(pl, 0, pl.nin, pl.Pin, t, &w, t == pl.Lin - 1 ? sm.plan.vend : nullptr, bin_in);
        sm.tab_w[t] = w;
        sm.tab_w32[t] = (float)w;
    }
    for (int t = lane; t < pl.Lmid; t += 32) {
        double w;
        sm.tab_fm[t] = gray_entry(pl, pl.nin, pl.nmid, pl.Pmid, t, &w, nullptr, bin_mid);
        sm.tab_wm[t] = w;
    }
}

// Sum of the warp's lane accumulators (all lanes of a thread position hold the same total), times the
// scale, into sm.P.
template <int KH, int TPL, class WS>
__device__ __forceinline__ void reduce_warp_to_P(double (&ar)[KH], double (&ai)[KH], WS& sm, int c0) {
    const int lane = threadIdx.x & 31;
    __syncwarp();
#pragma unroll
    for (int j = 0; j < KH; ++j) {
#pragma unroll
        for (int o = TPL; o < 32; o <<= 1) {
            ar[j] += __shfl_xor_sync(0xffffffffu, ar[j], o);
            ai[j] += __shfl_xor_sync(0xffffffffu, ai[j], o);
        }
    }
    if (lane < TPL) {
#pragma unroll
        for (int j = 0; j < KH; ++j)
            if (c0 + j < sm.plan.K) sm.P[c0 + j] = make_double2(ar[j] * sm.plan.scale, ai[j] * sm.plan.scale);
    }
    __syncwarp();
}

template <int KP, int TPL, class WS>
__device__ void sweep_warp_f64(WS& sm) {
    constexpr int KH = KP / TPL;
    const auto& pl = sm.plan;
    const int lane_id = threadIdx.x & 31;
    const int lanes = 32 / TPL, lane = lane_id / TPL, h = lane_id % TPL, c0 = h * KH;
    const unsigned gmask = 0xffffffffu;                    // the warp walks its lanes in lockstep
    const int K = pl.K, Lin = pl.Lin, Lmid = pl.Lmid, nin = pl.nin;
    const int64_t H = pl.H;
    double ar[KH], ai[KH];
#pragma unroll
    for (int j = 0; j < KH; ++j) { ar[j] = 0.0; ai[j] = 0.0; }
    for (int64_t hw = 0; hw < H; hw += lanes) {
        double sr[KH], si[KH], wh;
        int64_t hl = hw + lane;
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
            inner_block<KH, TPL, 1, double, double2, double>(sr, si, ar, ai, sm, sm.B, sm.tab_w, wmh, 2.0, !(pm & 1),
                                                             Lin, c0, h, gmask);
        }
    }
    reduce_warp_to_P<KH, TPL>(ar, ai, sm, c0);
}

template <int KP, int TPL, class WS>
__device__ void sweep_warp_mixed(WS& sm) {
    constexpr int KH = KP / TPL;
    const auto& pl = sm.plan;
    const int lane_id = threadIdx.x & 31;
    const int lanes = 32 / TPL, lane = lane_id / TPL, h = lane_id % TPL, c0 = h * KH;
    const unsigned gmask = 0xffffffffu;
    const int K = pl.K, Lin = pl.Lin, Lmid = pl.Lmid;
    const int64_t H = pl.H;
    double ar[KH], ai[KH];
#pragma unroll
    for (int j = 0; j < KH; ++j) { ar[j] = 0.0; ai[j] = 0.0; }
    for (int64_t hw = 0; hw < H; hw += lanes) {
        double wh;
        int64_t hl = hw + lane;
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
            float a32r[KH], a32i[KH];
#pragma unroll
            for (int j = 0; j < KH; ++j) { a32r[j] = 0.0f; a32i[j] = 0.0f; }
            inner_block<KH, TPL, 1, float, float2, float>(sr, si, a32r, a32i, sm, sm.B32, sm.tab_w32, 1.0f, 1.0f, fwd,
                                                          Lin, c0, h, gmask);
            const double wmh = wh * sm.tab_wm[pm];
#pragma unroll
            for (int j = 0; j < KH; ++j) { ar[j] = fma(wmh, (double)a32r[j], ar[j]); ai[j] = fma(wmh, (double)a32i[j], ai[j]); }
        }
    }
    reduce_warp_to_P<KH, TPL>(ar, ai, sm, c0);
}

#define PE_WTIER(KPv, CALL)                                  \
    if constexpr (KPW >= KPv) {                              \
        if (K <= KPv) { CALL; return; }                      \
    }

template <int TPL, int KPW, bool MIXED, class WS>
__device__ void warp_cofactors(WS& sm, int K) {
    if constexpr (MIXED) {
        PE_WTIER(4, (sweep_warp_mixed<4, TPL>(sm)))
        PE_WTIER(8, (sweep_warp_mixed<8, TPL>(sm)))
        PE_WTIER(12, (sweep_warp_mixed<12, TPL>(sm)))
        PE_WTIER(16, (sweep_warp_mixed<16, TPL>(sm)))
    } else {
        PE_WTIER(4, (sweep_warp_f64<4, TPL>(sm)))
        PE_WTIER(8, (sweep_warp_f64<8, TPL>(sm)))
        PE_WTIER(12, (sweep_warp_f64<12, TPL>(sm)))
        PE_WTIER(16, (sweep_warp_f64<16, TPL>(sm)))
    }
}

// Marginal, CDF and pick of one step (the rule of cofactors_triton.py:298-308, tot = cw[m - 1]); the
// 32-mode chunks are scanned twice.  Returns min |cw - u tot| / tot.
template <int DRW, class WS>
static __device__ double draw_warp_chunks(WS& sm, const double2* __restrict__ A, int m, int k, double u,
                                          double* __restrict__ marg_row) {
    const int lane = threadIdx.x & 31;
    double tot = 0.0;
    for (int pass = 0; pass < 2; ++pass) {
        const double target = u * tot;
        double carry = 0.0, gmin = 1.0e300;
        int cnt = 0;
        // DRW chunks of 32 modes at a time: DRW independent loads in flight per column and lane (the
        // amplitudes are the same sums in the same order; the chunks are then scanned one after another)
        for (int base = 0; base < m; base += 32 * DRW) {
            double xr[DRW], xi[DRW];
#pragma unroll
            for (int r = 0; r < DRW; ++r) { xr[r] = 0.0; xi[r] = 0.0; }
#pragma unroll 2
            for (int c = 0; c < k; ++c) {
                const int64_t co = (int64_t)sm.cols[c] * m;
                const double2 p = sm.P[c];
                double2 a[DRW];
#pragma unroll
                for (int r = 0; r < DRW; ++r) {
                    const int rho = base + 32 * r + lane;
                    a[r] = rho < m ? A[(int64_t)rho + co] : make_double2(0.0, 0.0);
                }
#pragma unroll
                for (int r = 0; r < DRW; ++r) {
                    xr[r] = fma(a[r].x, p.x, xr[r]);
                    xr[r] = fma(-a[r].y, p.y, xr[r]);
                    xi[r] = fma(a[r].x, p.y, xi[r]);
                    xi[r] = fma(a[r].y, p.x, xi[r]);
                }
            }
#pragma unroll
            for (int r = 0; r < DRW; ++r) {
                const int rho = base + 32 * r + lane;
                const double w = rho < m ? xr[r] * xr[r] + xi[r] * xi[r] : 0.0;
                double x = w;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const double y = __shfl_up_sync(0xffffffffu, x, o);
                    if (lane >= o) x += y;
                }
                const double cw = carry + x;
                if (pass == 1 && rho < m) {
                    cnt += (cw < target) ? 1 : 0;
                    gmin = fmin(gmin, fabs(cw - target));
                    if (marg_row) marg_row[rho] = w / tot;
                }
                carry = __shfl_sync(0xffffffffu, cw, 31);
            }
        }
        if (pass == 0) {
            tot = carry;
        } else {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
                gmin = fmin(gmin, __shfl_xor_sync(0xffffffffu, gmin, o));
            }
            if (lane == 0) sm.rows[k - 1] = min(cnt, m - 1);
            __syncwarp();
            return gmin / tot;
        }
    }
    return 0.0;
}

// The same draw for at most 32 NCH modes in one pass: every chunk's amplitudes at once (NCH loads of A in
// flight per column and lane, the columns four at a time), the cumulative weights kept in registers for the
// pick.  Same sums, scans and comparisons as draw_warp_chunks, so the same bits and the same pick.
template <int NCH, class WS>
static __device__ double draw_warp_regs(WS& sm, const double2* __restrict__ A, int m, int k, double u,
                                        double* __restrict__ marg_row) {
    const int lane = threadIdx.x & 31;
    const int nch = (m + 31) >> 5;
    double xr[NCH], xi[NCH];
#pragma unroll
    for (int r = 0; r < NCH; ++r) { xr[r] = 0.0; xi[r] = 0.0; }
#pragma unroll 4
    for (int c = 0; c < k; ++c) {
        const int64_t co = (int64_t)sm.cols[c] * m;
        const double2 p = sm.P[c];
        double2 a[NCH];
#pragma unroll
        for (int r = 0; r < NCH; ++r) {
            const int rho = 32 * r + lane;
            a[r] = (r < nch && rho < m) ? A[(int64_t)rho + co] : make_double2(0.0, 0.0);
        }
#pragma unroll
        for (int r = 0; r < NCH; ++r) {
            xr[r] = fma(a[r].x, p.x, xr[r]);
            xr[r] = fma(-a[r].y, p.y, xr[r]);
            xi[r] = fma(a[r].x, p.y, xi[r]);
            xi[r] = fma(a[r].y, p.x, xi[r]);
        }
    }
    double w[NCH], cw[NCH];
    double carry = 0.0;
#pragma unroll
    for (int r = 0; r < NCH; ++r) {
        const int rho = 32 * r + lane;
        w[r] = rho < m ? xr[r] * xr[r] + xi[r] * xi[r] : 0.0;
        cw[r] = 0.0;
        if (r < nch) {
            double x = w[r];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const double y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            cw[r] = carry + x;
            carry = __shfl_sync(0xffffffffu, cw[r], 31);
        }
    }
    const double tot = carry, target = u * tot;
    int cnt = 0;
    double gmin = 1.0e300;
#pragma unroll
    for (int r = 0; r < NCH; ++r) {
        const int rho = 32 * r + lane;
        if (r < nch && rho < m) {
            cnt += (cw[r] < target) ? 1 : 0;
            gmin = fmin(gmin, fabs(cw[r] - target));
            if (marg_row) marg_row[rho] = w[r] / tot;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        gmin = fmin(gmin, __shfl_xor_sync(0xffffffffu, gmin, o));
    }
    if (lane == 0) sm.rows[k - 1] = min(cnt, m - 1);
    __syncwarp();
    return gmin / tot;
}

// Weights and inclusive CDF of one piece of 32 DRW modes from `carry` (the CDF before the piece), as
// draw_warp_chunks forms them; returns the CDF at the piece's end.
template <int DRW, class WS>
static __device__ __forceinline__ double draw_piece(const WS& sm, const double2* __restrict__ A, int m, int k,
                                                    int base, double carry, double (&w)[DRW], double (&cw)[DRW]) {
    const int lane = threadIdx.x & 31;
    double xr[DRW], xi[DRW];
#pragma unroll
    for (int r = 0; r < DRW; ++r) { xr[r] = 0.0; xi[r] = 0.0; }
#pragma unroll 2
    for (int c = 0; c < k; ++c) {
        const int64_t co = (int64_t)sm.cols[c] * m;
        const double2 p = sm.P[c];
        double2 a[DRW];
#pragma unroll
        for (int r = 0; r < DRW; ++r) {
            const int rho = base + 32 * r + lane;
            a[r] = rho < m ? A[(int64_t)rho + co] : make_double2(0.0, 0.0);
        }
#pragma unroll
        for (int r = 0; r < DRW; ++r) {
            xr[r] = fma(a[r].x, p.x, xr[r]);
            xr[r] = fma(-a[r].y, p.y, xr[r]);
            xi[r] = fma(a[r].x, p.y, xi[r]);
            xi[r] = fma(a[r].y, p.x, xi[r]);
        }
    }
#pragma unroll
    for (int r = 0; r < DRW; ++r) {
        const int rho = base + 32 * r + lane;
        w[r] = rho < m ? xr[r] * xr[r] + xi[r] * xi[r] : 0.0;
        double x = w[r];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        cw[r] = carry + x;
        carry = __shfl_sync(0xffffffffu, cw[r], 31);
    }
    return carry;
}

// The draw for 129 to 4096 modes without a second full pass: the first pass keeps the CDF at the end of
// every 128-mode piece (piece p in lane p), the pick's piece is the first whose end reaches u tot, and only
// that piece is formed again (the same sums from the same carry, so the same bits).  The CDF grows
// monotonically from piece to piece (non-negative weights added to the carry), so every mode of an earlier
// piece lies below u tot and none of a later one does: the count, and the distance of the CDF to u tot
// (at the pick's piece and at the end of the piece before it), are those of the full scan.
template <class WS>
static __device__ double draw_warp_pieces(WS& sm, const double2* __restrict__ A, int m, int k, double u) {
    constexpr int DRW = 4, PIECE = 32 * DRW;
    const int lane = threadIdx.x & 31;
    const int np = (m + PIECE - 1) / PIECE;
    double w[DRW], cw[DRW];
    double carry = 0.0, mine = 0.0;
    for (int pc = 0; pc < np; ++pc) {
        carry = draw_piece<DRW>(sm, A, m, k, pc * PIECE, carry, w, cw);
        if (lane == pc) mine = carry;
    }
    const double tot = carry, target = u * tot;
    const unsigned reach = __ballot_sync(0xffffffffu, lane < np && mine >= target);
    const int j = reach ? __ffs(reach) - 1 : np - 1;
    const double prev = __shfl_sync(0xffffffffu, mine, j > 0 ? j - 1 : 0);
    draw_piece<DRW>(sm, A, m, k, j * PIECE, j > 0 ? prev : 0.0, w, cw);
    int cnt = 0;
    double gmin = j > 0 ? fabs(prev - target) : 1.0e300;
#pragma unroll
    for (int r = 0; r < DRW; ++r) {
        const int rho = j * PIECE + 32 * r + lane;
        if (rho < m) {
            cnt += (cw[r] < target) ? 1 : 0;
            gmin = fmin(gmin, fabs(cw[r] - target));
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        gmin = fmin(gmin, __shfl_xor_sync(0xffffffffu, gmin, o));
    }
    if (lane == 0) sm.rows[k - 1] = min(j * PIECE + cnt, m - 1);
    __syncwarp();
    return gmin / tot;
}

// Up to 128 modes in one pass with the weights in registers (two chunks' registers up to 64 modes); up to
// 4096 in 128-mode pieces with only the pick's piece formed twice; beyond, or when the marginal itself is
// asked for, the whole CDF scanned twice (L2 latency hidden by four chunks' independent loads).
template <class WS>
static __device__ double draw_warp(WS& sm, const double2* __restrict__ A, int m, int k, double u,
                                   double* __restrict__ marg_row) {
    if (m <= 64) return draw_warp_regs<2>(sm, A, m, k, u, marg_row);
    if (m <= 128) return draw_warp_regs<4>(sm, A, m, k, u, marg_row);
    if (!marg_row && m <= 32 * 128) return draw_warp_pieces(sm, A, m, k, u);
    return draw_warp_chunks<4>(sm, A, m, k, u, marg_row);
}

template <int TPL, int KPW, bool MIXED, class WS>
__device__ void chain_warp(const ChainParams& p, WS& sm, int64_t s) {
    const int lane = threadIdx.x & 31;
    const int64_t g = p.dp[s];
    bool ok = g >= 0 && g < p.G;
    int m = 0, nin = 0;
    int64_t off = 0;
    if (ok) { m = p.inst_m[g]; nin = p.inst_n[g]; off = p.inst_off[g]; }
    const int nk = p.nk ? p.nk[s] : p.n_stride;
    const int kf = p.k_first;
    if (nk < kf - 1) return;                                  // nothing to run (a dropped stream)
    ok = ok && nk >= 0 && nk <= p.n_stride && nk <= KPW && m >= 1 && m <= p.m_cap && m <= p.occ_stride;
    bool bad = false;
    if (ok && lane < nk) {
        const int64_t c = p.cols[s * p.n_stride + lane];
        if (c < 0 || c >= nin) bad = true;
        else sm.cols[lane] = (int)c;
    }
    if (ok && lane < kf - 1) {
        const int64_t r = p.rows[s * p.n_stride + lane];
        if (r < 0 || r >= m) bad = true;
        else sm.rows[lane] = (int)r;
    }
    if (!ok || __any_sync(0xffffffffu, bad)) {
        if (lane == 0) record_error(p.status, p.detail, s);
        __syncwarp();
        return;
    }
    build_groups_warp(sm, kf - 1);
    if (lane == 0) { sm.lane0 = 0; sm.lane_mult = 1; }
    __syncwarp();
    const double2* A = p.acol + off;
    const int kend = (p.k_stop > 0 && p.k_stop < nk) ? p.k_stop : nk;
    for (int k = kf; k <= kend; ++k) {
        const int K1 = k - 1;
        if (K1 == 0) {
            if (lane == 0) sm.P[0] = make_double2(1.0, 0.0);
            __syncwarp();
        } else {
            plan_step(sm, K1, k, 32 / TPL, WLIN, WMID);
            __syncwarp();
            prepare_warp(sm, A, m, MIXED);
            __syncwarp();
            warp_cofactors<TPL, KPW, MIXED>(sm, k);
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
        const double gap = draw_warp(sm, A, m, k, u, mrow);
        if constexpr (MIXED) {
            if (K1 > 0 && gap <= guard_band(p, k)) {       // guard band: this step again in FP64
                warp_cofactors<TPL, KPW, false>(sm, k);
                draw_warp(sm, A, m, k, u, mrow);
            }
        }
        if (lane == 0) add_to_groups(sm, sm.rows[k - 1]);
        __syncwarp();
    }
    for (int j = kf - 1 + lane; j < kend; j += 32) p.rows[s * p.n_stride + j] = sm.rows[j];
    if (p.occ && kend == nk) {
        for (int rho = lane; rho < p.occ_stride; rho += 32) {
            int c = 0;
            for (int j = 0; j < nk; ++j) c += (sm.rows[j] == rho) ? 1 : 0;
            p.occ[s * (int64_t)p.occ_stride + rho] = c;
        }
    }
    __syncwarp();
}

// Two-thread lanes of at most 8 columns fit 80 registers and a 5 KB slice per stream: three CTAs per SM
// (24 streams in flight instead of 16); the others keep two.
template <int TPL, int KPW>
constexpr int warp_ctas_per_sm() { return (KPW <= 8 && TPL == 2) ? 3 : 2; }

template <int TPL, int KPW, bool MIXED>
__global__ void __launch_bounds__(32 * WARPS, warp_ctas_per_sm<TPL, KPW>()) fock_chain_warp_kernel(ChainParams p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using WS = WarpSmemT<KPW>;
    WS& sm = reinterpret_cast<WS*>(smem_raw)[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    for (;;) {
        if (lane == 0) {
            sm.cur = queue_stream(p, atomicAdd(p.queue, 1ull));
        }
        __syncwarp();
        const int64_t s = sm.cur;
        if (s < 0) return;
        if (s >= p.S) {
            if (lane == 0) record_error(p.status, p.detail, s);
            return;
        }
        chain_warp<TPL, KPW, MIXED>(p, sm, s);
    }
}

}  // namespace pe
