// Device building blocks of the Fock chain kernels: Philox uniforms, exact signed binomials and the
// per-CTA shared-memory layout.  sm_100a only.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pe {

constexpr int MAXN = 64;        // photons per stream = largest cofactor tier (columns)
constexpr int NARROW = 32;      // tiers up to this many columns keep 32-wide shared-memory tables
constexpr int LIN_MAX = 512;    // inner Gray block: terms walked from the shared inner schedule
constexpr int MID_MAX = 1024;   // middle Gray block: inner blocks walked from the shared middle schedule
constexpr int MAX_WARPS = 8;    // CTA of at most 256 threads

// ------------------------------------------------------------------------------------------ RNG
// Philox4x32-10 with the counter/key arrangement of Triton's tl.rand for an int32 offset and a
// seed below 2^31 (triton/language/random.py: randint4x -> philox -> philox_impl): counter
// (offset, 0, 0, 0), key (seed_lo, seed_hi), first output word.
static __device__ __forceinline__ uint32_t philox_word0(uint64_t seed, uint32_t offset) {
    uint32_t c0 = offset, c1 = 0u, c2 = 0u, c3 = 0u;
    uint32_t k0 = (uint32_t)(seed & 0xffffffffull), k1 = (uint32_t)(seed >> 32);
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t o0 = c0, o2 = c2;
        c0 = __umulhi(0xCD9E8D57u, o2) ^ c1 ^ k0;
        c2 = __umulhi(0xD2511F53u, o0) ^ c3 ^ k1;
        c1 = 0xCD9E8D57u * o2;
        c3 = 0xD2511F53u * o0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c0;
}

// tl.rand: the word as int32, negatives folded to -x - 1, times float32(4.6566127342e-10), in f32.
static __device__ __forceinline__ float triton_uniform_f32(uint64_t seed, uint32_t offset) {
    int32_t x = (int32_t)philox_word0(seed, offset);
    if (x < 0) x = -x - 1;
    return __fmul_rn(__int2float_rn(x), 4.6566127342e-10f);
}

// The draw kernel's 48-bit uniform of stream-offset `off`: (r0 + r1 2^-24) / (1 + 2^-24), f64.
static __device__ __forceinline__ double chain_uniform(uint64_t seed, int64_t off) {
    const double r0 = (double)triton_uniform_f32(seed, (uint32_t)(2 * off));
    const double r1 = (double)triton_uniform_f32(seed, (uint32_t)(2 * off + 1));
    const double num = __dadd_rn(r0, __dmul_rn(r1, 5.9604644775390625e-08));
    return __ddiv_rn(num, 1.0 + 5.9604644775390625e-08);
}

// ------------------------------------------------------------------------------------------ maths
// (-1)^v C(M, v), exact: the integer product is formed in int64 (M <= 32) before conversion.
static __device__ __forceinline__ double signed_binom(int M, int v) {
    if (v == 0) return 1.0;                          // the usual multiplicities without 64-bit divisions
    if (v == 1) return -(double)M;
    if (v == 2) return (double)(M * (M - 1) / 2);
    int64_t c = 1;
    for (int i = 0; i < v; ++i) c = c * (M - i) / (i + 1);
    return (v & 1) ? -(double)c : (double)c;
}

// ------------------------------------------------------------------------------------------ layout
// Per-step plan of one stream.  The collapsed sum runs over v in prod_d {0..R_d - 1}; its digits are
// ordered for the kernel as
//   [inner: nin | middle: nmid | high: nhi | fixed]
// inner digits are walked from the shared inner schedule (one CTA-uniform transition per term),
// middle digits from the shared middle schedule once per inner block, high digits index the Gray
// lanes (each lane owns one combination of them), fixed digits have radix 1.
template <int NK>
struct PlanT {
    static constexpr int NKMAX = NK;   // largest number of columns (and of row groups + 1) it holds
    int64_t N;          // terms of the collapsed sum (the reference's addend count)
    int64_t H;          // lanes = product of high radices
    int Lin, Lmid;      // inner / middle combinations
    int K, K1, D;       // columns, chosen rows, digits (distinct chosen rows)
    int nin, nmid, nhi;
    double scale;       // 2^-K1, doubled when an odd group is halved
    int R[NK];        // radix per kernel digit
    int M[NK];        // multiplicity per kernel digit
    int drow[NK];     // output mode per kernel digit
    int Pin[NK];      // prefix products of the inner radices
    int Pmid[NK];     // prefix products of the middle radices
    unsigned char vend[NK];   // inner digit values after a forward inner block
    int sortR[NK];    // scratch of the planner: active digits by ascending radix
    int sortG[NK];
};

// Shared memory of one CTA working on one stream, for tiers of up to NK columns (32: the narrow layout
// of chains up to 32 photons; 64: the wide one, FP64 only, so its FP32 copy of B is a placeholder).
// COMP: the compensated form's layout, with the low parts of 2B beside the high ones.
template <int NK, bool COMP = false>
struct SmemT {
    static constexpr int NKMAX = NK;
    static constexpr int NK32 = NK <= NARROW ? NK : 1;
    static constexpr int NKLO = COMP ? NK32 : 1;
    PlanT<NK> plan;
    double2 P[NK];                 // cofactors of the step (scaled)
    double2 B[NK][NK];             // B[kd][j] = A[drow_kd, col_j], padded columns zero
    alignas(16) float2 B32[NK32][NK32];   // 2 * B in float32 (the mixed form's Gray update); paired
                                   // sweeps read each row as float4 slots (see prepare_step)
    alignas(16) float2 B32lo[NKLO][NKLO];  // compensated form: 2B - B32 (B32 then lies on the grid)
    double grid;                   // compensated form: power-of-two grid of the column sums' high parts
    double tab_w[LIN_MAX];         // inner weight prod (-1)^v C(M, v) at inner index t
    float tab_w32[LIN_MAX];
    double tab_wm[MID_MAX];        // middle weight at middle index
    unsigned char tab_f[LIN_MAX];  // transition into inner index t: digit | 0x80 when the update is -2 b
    unsigned char tab_fm[MID_MAX]; // transition into middle index: middle digit | 0x80 when -2 b
    double2 red[MAX_WARPS][NK];  // cross-warp reduction
    double scan[MAX_WARPS];
    double fmin[MAX_WARPS];
    int cnt[MAX_WARPS];
    int rows[NK];                // chosen modes so far
    int cols[NK];                // input columns of the stream in chain order
    int grow[NK];                // distinct chosen modes (groups), in order of first appearance
    int gmul[NK];                // their multiplicities
    int ngrp;
    int64_t cur;                   // stream being processed (-1: queue drained)
    int64_t lane0;                 // this CTA's first Gray lane (split steps: chunk * lanes)
    int lane_mult;                 // CTAs sharing one step of a stream (1 unless the step is split)
    double tot, target;
    int bad;                       // set by any thread that saw an out-of-range index
};

// Precision forms (the values of PE_PRECISION_* in pe_b200.h)
constexpr int PREC_F64 = 0, PREC_MIXED = 1, PREC_COMP = 2;

using Plan = PlanT<NARROW>;
using Smem = SmemT<NARROW>;
template <int KPM, int PREC = PREC_F64>
using SmemFor = SmemT<(KPM <= NARROW ? NARROW : MAXN), PREC == PREC_COMP>;

// Dynamic shared memory of a chain CTA before its m weights: the layout of the tier, 16-byte rounded.
template <int KPM, int PREC = PREC_F64>
__host__ __device__ constexpr size_t smem_fixed_bytes() { return (sizeof(SmemFor<KPM, PREC>) + 15) & ~(size_t)15; }
__host__ __device__ constexpr size_t smem_fixed_bytes_for(int kpm, int prec = PREC_F64) {
    return kpm <= NARROW ? (prec == PREC_COMP ? smem_fixed_bytes<NARROW, PREC_COMP>() : smem_fixed_bytes<NARROW>())
                         : smem_fixed_bytes<MAXN>();
}

}  // namespace pe
