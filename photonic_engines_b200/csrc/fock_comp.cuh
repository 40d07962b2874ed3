// Compensated mixed-precision sweep: complex FP32 Gray blocks whose column sums, products and block
// accumulators are carried as unevaluated FP32 pairs (hi + lo), so that a block's sum is as accurate
// as an FP64 one while every operation issues on the FP32 pipe (paired FFMA2 / FMUL2 / FADD2).
//
//   column sums   s = sh + sl with sh on a power-of-two grid g chosen per step so that every column sum
//                 of the step is below 2^24 g: the Gray update sh += +-(2b)_hi is then exact in FP32, and
//                 the small remainders (2b)_lo accumulate in sl
//   products      error-free: p = a*b and e = fma(a, b, -p) (TwoProduct) for the four real products of a
//                 complex product, TwoSum for their difference / sum, first-order cross terms of the low
//                 parts with FMAs (double-float arithmetic without renormalisation)
//   accumulation  acc += term with TwoSum on the high parts, the errors and low parts into acc_lo
//   blocks        each inner block (at most 512 terms) starts from column sums formed in FP64 and is folded
//                 into FP64 accumulators (the cross-block Glynn sum), as the other sweeps do
//
// Included by fock_kernels.cuh after the FP64 and mixed sweeps (it uses lane_digits / lane_sums).
// The reference keeps the sweep in FP64 (photonic_engines/clifford/cuda_cofactors.py:35-151); its
// double-double building blocks are two_sum / two_prod in photonic_engines/gaussian/dd.py:1-60.
#pragma once

namespace pe {

// ---------------------------------------------------------------------------------------- paired FP32
static __device__ __forceinline__ float2 c_add(float2 a, float2 b) { return __fadd2_rn(a, b); }
static __device__ __forceinline__ float2 c_sub(float2 a, float2 b) {
    unsigned long long ra = *reinterpret_cast<unsigned long long*>(&a), rb = *reinterpret_cast<unsigned long long*>(&b), rd;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(rd) : "l"(ra), "l"(rb));
    return *reinterpret_cast<float2*>(&rd);
}
static __device__ __forceinline__ float2 c_mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
static __device__ __forceinline__ float2 c_fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
static __device__ __forceinline__ float2 c_neg(float2 a) { return make_float2(-a.x, -a.y); }

// A complex double-float value for two columns side by side (.x one column, .y the other).
struct CDF2 {
    float2 rh, ih, rl, il;
};

// z = x * y, both complex double-float (paired over two columns).  Real part: TwoProduct of xr*yr and
// xi*yi, TwoSum of their difference, then the product errors and the first-order low-part terms;
// imaginary part likewise.  The second-order low x low terms are below the pair's precision.
static __device__ __forceinline__ CDF2 cmul_cdf(const CDF2& x, const CDF2& y) {
    CDF2 z;
    {
        const float2 p1 = c_mul(x.rh, y.rh), e1 = c_fma(x.rh, y.rh, c_neg(p1));
        const float2 p2 = c_mul(x.ih, y.ih), e2 = c_fma(x.ih, y.ih, c_neg(p2));
        const float2 h = c_sub(p1, p2);
        const float2 bb = c_sub(h, p1);
        const float2 e3 = c_sub(c_sub(p1, c_sub(h, bb)), c_add(p2, bb));
        float2 l = c_add(c_sub(e1, e2), e3);
        l = c_fma(x.rh, y.rl, l);
        l = c_fma(x.rl, y.rh, l);
        l = c_fma(c_neg(x.ih), y.il, l);
        l = c_fma(c_neg(x.il), y.ih, l);
        z.rh = h;
        z.rl = l;
    }
    {
        const float2 q1 = c_mul(x.rh, y.ih), f1 = c_fma(x.rh, y.ih, c_neg(q1));
        const float2 q2 = c_mul(x.ih, y.rh), f2 = c_fma(x.ih, y.rh, c_neg(q2));
        const float2 g = c_add(q1, q2);
        const float2 cc = c_sub(g, q1);
        const float2 f3 = c_add(c_sub(q1, c_sub(g, cc)), c_sub(q2, cc));
        float2 m = c_add(c_add(f1, f2), f3);
        m = c_fma(x.rh, y.il, m);
        m = c_fma(x.rl, y.ih, m);
        m = c_fma(x.ih, y.rl, m);
        m = c_fma(x.il, y.rh, m);
        z.ih = g;
        z.il = m;
    }
    return z;
}

// acc += t (TwoSum on the high parts; the rounding error and t's low part go to the low part).
static __device__ __forceinline__ void acc_cdf(float2& ah, float2& al, float2 th, float2 tl) {
    const float2 s = c_add(ah, th);
    const float2 bb = c_sub(s, ah);
    const float2 e = c_add(c_sub(ah, c_sub(s, bb)), c_sub(th, bb));
    ah = s;
    al = c_add(al, c_add(e, tl));
}

// The same product on one complex double-float number (scalar FP32): the exchange between the threads
// of a lane multiplies whole-thread totals.
struct CDF1 {
    float rh, ih, rl, il;
};
static __device__ __forceinline__ CDF1 cmul_cdf1(const CDF1& x, const CDF1& y) {
    CDF1 z;
    {
        const float p1 = x.rh * y.rh, e1 = fmaf(x.rh, y.rh, -p1);
        const float p2 = x.ih * y.ih, e2 = fmaf(x.ih, y.ih, -p2);
        const float h = p1 - p2, bb = h - p1;
        const float e3 = (p1 - (h - bb)) - (p2 + bb);
        float l = (e1 - e2) + e3;
        l = fmaf(x.rh, y.rl, l);
        l = fmaf(x.rl, y.rh, l);
        l = fmaf(-x.ih, y.il, l);
        l = fmaf(-x.il, y.ih, l);
        z.rh = h;
        z.rl = l;
    }
    {
        const float q1 = x.rh * y.ih, f1 = fmaf(x.rh, y.ih, -q1);
        const float q2 = x.ih * y.rh, f2 = fmaf(x.ih, y.rh, -q2);
        const float g = q1 + q2, cc = g - q1;
        const float f3 = (q1 - (g - cc)) + (q2 - cc);
        float m = (f1 + f2) + f3;
        m = fmaf(x.rh, y.il, m);
        m = fmaf(x.rl, y.ih, m);
        m = fmaf(x.ih, y.rl, m);
        m = fmaf(x.il, y.rh, m);
        z.ih = g;
        z.il = m;
    }
    return z;
}
static __device__ __forceinline__ CDF1 shfl_cdf1(const CDF1& v, int o, unsigned gmask) {
    return {__shfl_xor_sync(gmask, v.rh, o), __shfl_xor_sync(gmask, v.ih, o), __shfl_xor_sync(gmask, v.rl, o),
            __shfl_xor_sync(gmask, v.il, o)};
}
static __device__ __forceinline__ CDF1 cdf1_x(const CDF2& v) { return {v.rh.x, v.ih.x, v.rl.x, v.il.x}; }
static __device__ __forceinline__ CDF1 cdf1_y(const CDF2& v) { return {v.rh.y, v.ih.y, v.rl.y, v.il.y}; }

// ---------------------------------------------------------------------------------------- prepare
// All threads, after prepare_step: the step's grid g (a power of two with every column sum below 2^23 g:
// bound = sum_kd M_kd max_j max(|Re B|, |Im B|)) and 2B split into an on-grid FP32 high part (B32) and an
// FP32 remainder (B32lo), both in the paired layout: row kd, float4 slot q = h * ka + c holds (re b_j1,
// re b_j2, im b_j1, im b_j2) with j1 = h * kh + c and j2 = j1 + ka (ka = kh2 / 2, kh2 = kh rounded up to
// even; a j2 at or beyond the thread's kh columns is padding and holds zero).
template <class SM>
static __device__ void prepare_comp(SM& sm, int kh, int tpl) {
    const auto& pl = sm.plan;
    const int tid = threadIdx.x, T = blockDim.x;
    if (tid < 32) {
        double part = 0.0;
        for (int kd = tid; kd < pl.D; kd += 32) {
            double mx = 0.0;
            for (int j = 0; j < pl.K; ++j) mx = fmax(mx, fmax(fabs(sm.B[kd][j].x), fabs(sm.B[kd][j].y)));
            part += (double)pl.M[kd] * mx;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
        if (tid == 0) {
            int e = 0;
            frexp(part > 0.0 ? part : 1.0, &e);               // part < 2^e
            sm.grid = ldexp(1.0, e - 23);
        }
    }
    __syncthreads();
    const double g = sm.grid, ginv = 1.0 / g;                 // powers of two: exact
    const int kh2 = kh + (kh & 1), ka = kh2 / 2;
    const int slots = tpl * ka;                               // every thread's slots, padding included
    for (int idx = tid; idx < pl.D * slots; idx += T) {
        const int kd = idx / slots, q = idx % slots;
        const int h = q / ka, c = q % ka;
        const int j1 = h * kh + c, j2 = h * kh + ka + c;
        const bool v1 = j1 < pl.K, v2 = (ka + c) < kh && j2 < pl.K;
        const double2 b1 = v1 ? sm.B[kd][j1] : make_double2(0.0, 0.0);
        const double2 b2 = v2 ? sm.B[kd][j2] : make_double2(0.0, 0.0);
        const double r1 = rint(2.0 * b1.x * ginv) * g, i1 = rint(2.0 * b1.y * ginv) * g;
        const double r2 = rint(2.0 * b2.x * ginv) * g, i2 = rint(2.0 * b2.y * ginv) * g;
        reinterpret_cast<float4*>(&sm.B32[kd][0])[q] = make_float4((float)r1, (float)r2, (float)i1, (float)i2);
        reinterpret_cast<float4*>(&sm.B32lo[kd][0])[q] =
            make_float4((float)(2.0 * b1.x - r1), (float)(2.0 * b2.x - r2), (float)(2.0 * b1.y - i1),
                        (float)(2.0 * b2.y - i2));
    }
}

// ---------------------------------------------------------------------------------------- sweep
// One term over this thread's KA column pairs: optional exact Gray update (brow: high / low rows of 2B),
// prefix chain, suffix chain seeded with the other columns' product, compensated accumulation.
template <int KA, int TPL>
__device__ __forceinline__ void term_comp(CDF2 (&s)[KA], float2 (&arh)[KA], float2 (&aih)[KA], float2 (&arl)[KA],
                                          float2 (&ail)[KA], const float4* bhi, const float4* blo, float f,
                                          float wh, float wl, int h, unsigned gmask) {
    if (bhi) {
        const float2 ff = make_float2(f, f);
#pragma unroll
        for (int c = 0; c < KA; ++c) {
            const float4 b = bhi[c], l = blo[c];
            s[c].rh = c_fma(ff, make_float2(b.x, b.y), s[c].rh);   // exact: on the step's grid
            s[c].ih = c_fma(ff, make_float2(b.z, b.w), s[c].ih);
            s[c].rl = c_fma(ff, make_float2(l.x, l.y), s[c].rl);
            s[c].il = c_fma(ff, make_float2(l.z, l.w), s[c].il);
        }
    }
    CDF2 pre[KA];
    CDF2 x;
    x.rh = make_float2(h == 0 ? wh : 1.0f, 1.0f);
    x.rl = make_float2(h == 0 ? wl : 0.0f, 0.0f);
    x.ih = make_float2(0.0f, 0.0f);
    x.il = make_float2(0.0f, 0.0f);
#pragma unroll
    for (int c = 0; c < KA; ++c) {
        pre[c] = x;
        x = cmul_cdf(x, s[c]);
    }
    // suffix starts: (other half's total) x (the other threads' product)
    CDF2 y;
    if constexpr (TPL == 1) {
        y.rh = make_float2(x.rh.y, x.rh.x); y.ih = make_float2(x.ih.y, x.ih.x);
        y.rl = make_float2(x.rl.y, x.rl.x); y.il = make_float2(x.il.y, x.il.x);
    } else {
        const CDF1 tot = cmul_cdf1(cdf1_x(x), cdf1_y(x));
        CDF1 o = shfl_cdf1(tot, 1, gmask);
        if constexpr (TPL == 4) {
            o = cmul_cdf1(o, shfl_cdf1(tot, 2, gmask));
            o = cmul_cdf1(o, shfl_cdf1(tot, 3, gmask));
        }
        CDF2 sw, oo;
        sw.rh = make_float2(x.rh.y, x.rh.x); sw.ih = make_float2(x.ih.y, x.ih.x);
        sw.rl = make_float2(x.rl.y, x.rl.x); sw.il = make_float2(x.il.y, x.il.x);
        oo.rh = make_float2(o.rh, o.rh); oo.ih = make_float2(o.ih, o.ih);
        oo.rl = make_float2(o.rl, o.rl); oo.il = make_float2(o.il, o.il);
        y = cmul_cdf(sw, oo);
    }
#pragma unroll
    for (int c = KA - 1; c >= 0; --c) {
        const CDF2 t = cmul_cdf(pre[c], y);
        acc_cdf(arh[c], arl[c], t.rh, t.rl);
        acc_cdf(aih[c], ail[c], t.ih, t.il);
        if (c > 0) y = cmul_cdf(y, s[c]);
    }
}

// Compensated sweep of tier KP.  A thread's KH = KP / TPL columns are held as KA = ceil(KH / 2) pairs
// (column c and KA + c of the thread); a pair slot beyond the thread's columns, and columns beyond K,
// have column sum 1 and zero updates.
template <int KP, int TPL, class SM>
__device__ void sweep_comp(SM& sm) {
    constexpr int KH = KP / TPL;
    constexpr int KA = (KH + 1) / 2;
    const auto& pl = sm.plan;
    const int tid = threadIdx.x;
    const int lanes = blockDim.x / TPL, lane = tid / TPL, h = tid % TPL, c0 = h * KH;
    const int wl0 = (tid & ~31) / TPL;
    const unsigned gmask = 0xffffffffu;
    const int K = pl.K, Lin = pl.Lin, Lmid = pl.Lmid;
    const int64_t H = pl.H;
    const double g = sm.grid, ginv = 1.0 / g;
    double ar[2 * KA], ai[2 * KA];
#pragma unroll
    for (int j = 0; j < 2 * KA; ++j) { ar[j] = 0.0; ai[j] = 0.0; }
    for (int64_t hw = sm.lane0 + wl0; hw < H; hw += (int64_t)lanes * sm.lane_mult) {
        double wlane;
        int64_t hl = hw + (lane - wl0);
        const bool live = hl < H;
        if (!live) hl = H - 1;
        const uint64_t hpack = lane_digits(pl, hl, &wlane);
        if (!live) wlane = 0.0;
        for (int pm = 0; pm < Lmid; ++pm) {
            const bool fwd = !(pm & 1);
            CDF2 s[KA];
            {
                double xr[KH], xi[KH];
                lane_sums<KH>(sm, c0, !fwd, pm, hl, hpack, xr, xi);
                float sh[2][KA], si_[2][KA], lr[2][KA], li[2][KA];
#pragma unroll
                for (int q = 0; q < 2 * KA; ++q) {
                    const int half = q / KA, c = q % KA;
                    const bool pad = q >= KH || c0 + q >= K;
                    const double vr = pad ? 1.0 : xr[q < KH ? q : 0], vi = pad ? 0.0 : xi[q < KH ? q : 0];
                    const double hr = rint(vr * ginv) * g, hi = rint(vi * ginv) * g;
                    sh[half][c] = pad ? 1.0f : (float)hr;
                    si_[half][c] = pad ? 0.0f : (float)hi;
                    lr[half][c] = pad ? 0.0f : (float)(vr - hr);
                    li[half][c] = pad ? 0.0f : (float)(vi - hi);
                }
#pragma unroll
                for (int c = 0; c < KA; ++c) {
                    s[c].rh = make_float2(sh[0][c], sh[1][c]);
                    s[c].ih = make_float2(si_[0][c], si_[1][c]);
                    s[c].rl = make_float2(lr[0][c], lr[1][c]);
                    s[c].il = make_float2(li[0][c], li[1][c]);
                }
            }
            float2 arh[KA], aih[KA], arl[KA], ail[KA];
#pragma unroll
            for (int c = 0; c < KA; ++c) {
                arh[c] = make_float2(0.0f, 0.0f); aih[c] = arh[c]; arl[c] = arh[c]; ail[c] = arh[c];
            }
            const float4* bh = reinterpret_cast<const float4*>(&sm.B32[0][0]);
            const float4* bl = reinterpret_cast<const float4*>(&sm.B32lo[0][0]);
            constexpr int ROW = SM::NK32 / 2;                   // float4 slots per row
            const int q0 = h * KA;
            auto weight = [&](int t, float& whi, float& wlo) {
                const double w = sm.tab_w[t];
                whi = (float)w;
                wlo = (float)(w - (double)whi);
            };
            float whi, wlo;
            if (fwd) {
                weight(0, whi, wlo);
                term_comp<KA, TPL>(s, arh, aih, arl, ail, nullptr, nullptr, 0.0f, whi, wlo, h, gmask);
                for (int t = 1; t < Lin; ++t) {
                    const unsigned e = sm.tab_f[t];
                    weight(t, whi, wlo);
                    const int r = (int)(e & 63u) * ROW + q0;
                    term_comp<KA, TPL>(s, arh, aih, arl, ail, bh + r, bl + r, (e & 0x80u) ? -1.0f : 1.0f, whi, wlo,
                                       h, gmask);
                }
            } else {
                weight(Lin - 1, whi, wlo);
                term_comp<KA, TPL>(s, arh, aih, arl, ail, nullptr, nullptr, 0.0f, whi, wlo, h, gmask);
                for (int t = Lin - 2; t >= 0; --t) {
                    const unsigned e = sm.tab_f[t + 1];
                    weight(t, whi, wlo);
                    const int r = (int)(e & 63u) * ROW + q0;
                    term_comp<KA, TPL>(s, arh, aih, arl, ail, bh + r, bl + r, (e & 0x80u) ? 1.0f : -1.0f, whi, wlo,
                                       h, gmask);
                }
            }
            const double wmh = wlane * sm.tab_wm[pm];
#pragma unroll
            for (int c = 0; c < KA; ++c) {
                ar[c] = fma(wmh, (double)arh[c].x + (double)arl[c].x, ar[c]);
                ai[c] = fma(wmh, (double)aih[c].x + (double)ail[c].x, ai[c]);
                ar[KA + c] = fma(wmh, (double)arh[c].y + (double)arl[c].y, ar[KA + c]);
                ai[KA + c] = fma(wmh, (double)aih[c].y + (double)ail[c].y, ai[KA + c]);
            }
        }
    }
    // the first KH of the 2 KA accumulators are this thread's columns c0 .. c0 + KH - 1
    double rr[KH], ri[KH];
#pragma unroll
    for (int j = 0; j < KH; ++j) { rr[j] = ar[j]; ri[j] = ai[j]; }
    reduce_to_P<KH, TPL>(rr, ri, sm, c0);
}

template <int TPL, int KPM, class SM>
__device__ void dispatch_comp(SM& sm, int K) {
    PE_TIER(4, (sweep_comp<4, TPL>(sm)))
    PE_TIER(8, (sweep_comp<8, TPL>(sm)))
    PE_TIER(12, (sweep_comp<12, TPL>(sm)))
    PE_TIER(16, (sweep_comp<16, TPL>(sm)))
    PE_TIER(20, (sweep_comp<20, TPL>(sm)))
    PE_TIER(24, (sweep_comp<24, TPL>(sm)))
    PE_TIER(28, (sweep_comp<28, TPL>(sm)))
    PE_TIER(32, (sweep_comp<32, TPL>(sm)))
}

}  // namespace pe
