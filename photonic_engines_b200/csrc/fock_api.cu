// C ABI of the Fock chain kernels (declared in include/pe_b200.h): argument checks, variant
// lookup, occupancy-sized persistent grid, workspace reset, launch on the caller's stream.
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "fock_kernels.cuh"
#include "fock_registry.h"
#include "fock_warp.cuh"
#include "pe_errors.h"

namespace pe {

constexpr int N_KPM = 10;
constexpr int KPM_LADDER[N_KPM] = {8, 16, 20, 24, 28, 32, 40, 48, 56, 64};
static int kpm_for(int n) {
    for (int i = 0; i < N_KPM; ++i) if (n <= KPM_LADDER[i]) return KPM_LADDER[i];
    return -1;
}
static int tpl_index(int tpl) { return tpl == 1 ? 0 : tpl == 2 ? 1 : tpl == 4 ? 2 : -1; }
static int kpm_index(int kpm) {
    for (int i = 0; i < N_KPM; ++i) if (KPM_LADDER[i] == kpm) return i;
    return -1;
}

constexpr int N_PREC = 3;       // PE_PRECISION_F64, _MIXED, _COMPENSATED
static void* g_chain[N_PREC][3][N_KPM];
static void* g_cof[N_PREC][3][N_KPM];
static void* g_split_partial[N_PREC][3][N_KPM];
static void* g_split_draw[N_PREC][3][N_KPM];
static void* g_warp[N_PREC][3][N_KPM];
static size_t g_warp_slice[N_PREC][3][N_KPM];
static bool prec_ok(int p) { return p >= 0 && p < N_PREC; }

void register_variant(int mixed, int tpl, int kpm, void* chain_kernel, void* cofactor_kernel, void* split_partial,
                      void* split_draw, void* warp_kernel, size_t warp_slice_bytes) {
    const int ti = tpl_index(tpl), ki = kpm_index(kpm);
    if (!prec_ok(mixed) || ti < 0 || ki < 0) return;
    g_warp[mixed][ti][ki] = warp_kernel;
    g_warp_slice[mixed][ti][ki] = warp_slice_bytes;
    g_chain[mixed][ti][ki] = chain_kernel;
    g_cof[mixed][ti][ki] = cofactor_kernel;
    g_split_partial[mixed][ti][ki] = split_partial;
    g_split_draw[mixed][ti][ki] = split_draw;       // same launch bounds as the variant's other kernels
}
void* find_split_partial_kernel(int mixed, int tpl, int kpm) {
    const int ti = tpl_index(tpl), ki = kpm_index(kpm);
    return (!prec_ok(mixed) || ti < 0 || ki < 0) ? nullptr : g_split_partial[mixed][ti][ki];
}
void* find_warp_kernel(int mixed, int tpl, int kpm) {
    const int ti = tpl_index(tpl), ki = kpm_index(kpm);
    return (!prec_ok(mixed) || ti < 0 || ki < 0) ? nullptr : g_warp[mixed][ti][ki];
}
size_t warp_smem_bytes(int mixed, int tpl, int kpm, int warps) {
    const int ti = tpl_index(tpl), ki = kpm_index(kpm);
    const size_t slice = (!prec_ok(mixed) || ti < 0 || ki < 0) ? 0 : g_warp_slice[mixed][ti][ki];
    return (slice ? slice : sizeof(WarpSmem)) * (size_t)warps;
}
void* find_split_draw_kernel(int mixed, int tpl, int kpm) {
    const int ti = tpl_index(tpl), ki = kpm_index(kpm);
    return (!prec_ok(mixed) || ti < 0 || ki < 0) ? nullptr : g_split_draw[mixed][ti][ki];
}
void* find_chain_kernel(int mixed, int tpl, int kpm) {
    const int ti = tpl_index(tpl), ki = kpm_index(kpm);
    return (!prec_ok(mixed) || ti < 0 || ki < 0) ? nullptr : g_chain[mixed][ti][ki];
}
void* find_cofactor_kernel(int mixed, int tpl, int kpm) {
    const int ti = tpl_index(tpl), ki = kpm_index(kpm);
    return (!prec_ok(mixed) || ti < 0 || ki < 0) ? nullptr : g_cof[mixed][ti][ki];
}

// Threads per Gray lane when the caller passes 0 (measured at m = 400, 2 000 streams, and at m = 2n for
// 21-32 photons): one-thread lanes up to 8 columns, and for FP64 and mixed chains of 17-20 photons (no
// exchange of partial products; those variants run 128-thread CTAs with 255 registers: n = 20, m = 400,
// FP64 18.4 against 21.0 ms with two-thread lanes, mixed 12.8 against 13.4 ms); two-thread lanes beyond
// (at 24-40 columns compiled for 128-thread CTAs with 255 registers), four-thread lanes at 48-64.
static int default_tpl(int kpm, int precision) {
    if (kpm <= 8) return 1;
    if (precision != PE_PRECISION_COMPENSATED && kpm == 20) return 1;
    if (precision == PE_PRECISION_COMPENSATED) return kpm <= 20 ? 2 : 4;   // 12 FP32 pairs of state per column pair
    return kpm <= 40 ? 2 : 4;
}

static thread_local cudaError_t g_last_cuda_error = cudaSuccess;

int cuda_fail(cudaError_t e) {
    g_last_cuda_error = e;
    return PE_ERR_CUDA;
}

// Largest CTA a compiled kernel accepts (its launch bounds); 0 when the query fails (error recorded).
static int max_block(void* fn) {
    cudaFuncAttributes a;
    const cudaError_t e = cudaFuncGetAttributes(&a, fn);
    if (e != cudaSuccess) return cuda_fail(e), 0;
    return a.maxThreadsPerBlock;
}

static int max_smem_optin() {
    int dev = 0, v = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return cuda_fail(e), 0;
    return v;
}

// Arithmetic-pipe probe: 8 independent FMA chains per thread, `iters` rounds.  Used by the benchmark to
// measure the FP64 / FP32 peak of the GPU it runs on (the roofline denominator of the chain kernels).
template <typename T>
__global__ void pipe_probe_kernel(T* out, T a, T b, int iters) {
    T x[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) x[i] = (T)(threadIdx.x + i);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 8; ++i) x[i] = x[i] * a + b;
    }
    T s = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += x[i];
    out[(size_t)blockIdx.x * blockDim.x + threadIdx.x] = s;
}


// ---------------------------------------------------------------------------------------- adaptive
// Survivors of an adaptive chain (one CTA of 1024 threads).  col < 0: initial state, every stream alive.
// col >= 0: a live stream whose row rows[s][col] is an avoided mode is dropped.  Then nk[s] = n for the
// survivors and 0 for dropped streams (the chain kernels skip those), and rng[s] = the rank of s among
// the survivors of its pass chunk (chunk start s - off0[s]): the stream index the next step's draws use,
// because the reference shrinks the batch after every drop and renumbers the survivors
// (photonic_engines/clifford/sampler.py:436-446).  zero_dead: the occupation rows of dropped streams
// are cleared (the last update).
struct AvoidParams {
    const int64_t* rows;
    int n_stride;
    int col;
    const unsigned char* avoid;
    int m_max;
    unsigned char* alive;
    int32_t* nk;
    int64_t* rng;
    int64_t* scan;
    const int64_t* off0;
    int64_t S;
    int n;
    int64_t* occ;
    int occ_stride;
    int zero_dead;
    int* status;
    long long* detail;
};

__global__ void __launch_bounds__(1024) avoid_update_kernel(AvoidParams a) {
    __shared__ int64_t wsum[32];
    const int tid = threadIdx.x, T = blockDim.x, lid = tid & 31, wid = tid >> 5;
    for (int64_t s = tid; s < a.S; s += T) {
        int live = a.col < 0 ? 1 : a.alive[s];
        if (live && a.col >= 0) {
            const int64_t r = a.rows[s * a.n_stride + a.col];
            if (r < 0 || r >= a.m_max) { record_error(a.status, a.detail, s); live = 0; }
            else if (a.avoid[r]) live = 0;
        }
        a.alive[s] = (unsigned char)live;
        a.nk[s] = live ? a.n : 0;
        if (!live && a.zero_dead && a.occ)
            for (int rho = 0; rho < a.occ_stride; ++rho) a.occ[s * (int64_t)a.occ_stride + rho] = 0;
    }
    __syncthreads();
    // exclusive scan of alive: a contiguous chunk per thread, warp scan, warps in order
    const int64_t C = (a.S + T - 1) / T;
    const int64_t lo = min((int64_t)tid * C, a.S), hi = min(lo + C, a.S);
    int64_t loc = 0;
    for (int64_t i = lo; i < hi; ++i) loc += a.alive[i];
    int64_t x = loc;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lid >= o) x += y;
    }
    if (lid == 31) wsum[wid] = x;
    __syncthreads();
    int64_t base = x - loc;
    for (int w = 0; w < wid; ++w) base += wsum[w];
    for (int64_t i = lo; i < hi; ++i) { a.scan[i] = base; base += a.alive[i]; }
    __syncthreads();
    for (int64_t s = tid; s < a.S; s += T) {
        int64_t c = a.off0 ? s - a.off0[s] : 0;
        if (c < 0 || c > s) { record_error(a.status, a.detail, s); c = s; }
        a.rng[s] = a.scan[s] - a.scan[c];
    }
}

static size_t align16(size_t x) { return (x + 15) & ~(size_t)15; }
static size_t split_bytes(int64_t S, int nch) {
    return nch > 0 ? (size_t)S * nch * MAXN * sizeof(double2) + (size_t)S * sizeof(int) : 0;
}
}  // namespace pe

using namespace pe;

extern "C" int pe_version(void) { return 100; }

extern "C" int pe_max_modes(int block_threads) {
    (void)block_threads;
    const int cap = max_smem_optin();
    if (cap <= 0) return 0;
    return (int)((cap - (int)smem_fixed_bytes_for(NARROW)) / (int)sizeof(double));
}

extern "C" size_t pe_chain_workspace_bytes(int64_t S) {
    (void)S;
    return WS_BYTES;
}

extern "C" const char* pe_last_cuda_error(void) {
    return g_last_cuda_error == cudaSuccess ? "no CUDA error recorded" : cudaGetErrorString(g_last_cuda_error);
}

extern "C" const char* pe_status_string(int status) {
    switch (status) {
        case PE_OK: return "ok";
        case PE_ERR_ARG: return "invalid argument (null pointer, negative size or unknown option)";
        case PE_ERR_SIZE: return "size beyond the compiled limits (photons, modes or workspace)";
        case PE_ERR_CUDA: return "CUDA runtime error at launch";
        case PE_ERR_DEVICE: return "index out of range found on the device";
        default: return "unknown status";
    }
}

extern "C" int pe_read_status(const void* d_workspace, int* status, int64_t* detail, void* stream) {
    if (!d_workspace || !status) return PE_ERR_ARG;
    int st = 0;
    long long det = 0;
    cudaStream_t s = (cudaStream_t)stream;
    PE_CUDA_TRY(cudaMemcpyAsync(&st, (const char*)d_workspace + 8, sizeof(int), cudaMemcpyDeviceToHost, s));
    PE_CUDA_TRY(cudaMemcpyAsync(&det, (const char*)d_workspace + 16, sizeof(long long), cudaMemcpyDeviceToHost, s));
    PE_CUDA_TRY(cudaStreamSynchronize(s));
    *status = st;
    if (detail) *detail = (int64_t)det;
    return PE_OK;
}

static int launch_prepare(void* fn, int block, size_t smem, int* grid_per_sm) {
    PE_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int occ = 0;
    PE_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, block, smem));
    if (occ < 1) return PE_ERR_SIZE;
    *grid_per_sm = occ;
    return PE_OK;
}

// Checks, variant lookup and launches shared by the chain entry points.  k_split = 0: the whole chain in
// the persistent kernel; k_split >= 2: steps 1..k_split-1 there, then every step k >= k_split spread over
// nch CTAs per stream (split_partial) and drawn by one CTA per stream (split_draw).  Only the steps
// k_first..k_last run (k_last 0: to the end of every chain); rows[:, :k_first - 1] are read from d_rows.
// zero_status false keeps the status word of an earlier launch (the queue counter is always reset).
static int chain_launch(int precision, const double* d_acol, const int64_t* d_inst_off, const int32_t* d_inst_m,
                        const int32_t* d_inst_n, int G, int m_max, int64_t S, const int64_t* d_dp,
                        const int32_t* d_nk, const int64_t* d_cols, int n_stride, const double* d_uniforms,
                        const int64_t* d_seeds, const int64_t* d_seed_row, const int64_t* d_rng_off,
                        const int64_t* d_order, int64_t* d_rows, int64_t* d_occ, int occ_stride, double* d_marg,
                        int marg_stride, void* d_workspace, size_t workspace_bytes, int block_threads, int tpl,
                        int grid_ctas, int k_split, int nch, void* stream, bool warp_mode = false,
                        int k_first = 1, int k_last = 0, bool zero_status = true,
                        const int64_t* d_qrange = nullptr, int nk_max = 0, int64_t split_slots = 0) {
    if (!prec_ok(precision)) return PE_ERR_ARG;
    if (nk_max < 0 || nk_max > n_stride || split_slots < 0) return PE_ERR_ARG;
    if (d_qrange && k_split > 0 && split_slots < 1) return PE_ERR_ARG;      // a split range needs its slot count
    if (k_first < 1 || k_first > n_stride + 1 || k_last < 0) return PE_ERR_ARG;
    if (S < 0 || G < 1 || m_max < 1 || n_stride < 1) return PE_ERR_ARG;
    if (!d_acol || !d_inst_off || !d_inst_m || !d_inst_n || !d_dp || !d_cols || !d_rows || !d_workspace) return PE_ERR_ARG;
    if (!d_uniforms && !d_seeds) return PE_ERR_ARG;
    if (d_occ && occ_stride < m_max) return PE_ERR_ARG;
    if (d_marg && marg_stride < m_max) return PE_ERR_ARG;
    if (k_split < 0 || (k_split > 0 && (k_split < 2 || nch < 1))) return PE_ERR_ARG;
    const bool split = k_split > 0 && k_split <= n_stride;
    // split slots: every stream, or (a queue range) its first split_slots positions
    const int64_t nq = d_qrange ? (split_slots < S ? split_slots : S) : S;
    const size_t part_bytes = split ? (size_t)nq * nch * MAXN * sizeof(double2) : 0;
    const size_t need = WS_BYTES + part_bytes + (split ? (size_t)nq * sizeof(int) : 0);
    if (workspace_bytes < need || ((uintptr_t)d_workspace & 15u)) return PE_ERR_SIZE;
    const int ncols = nk_max > 0 ? nk_max : n_stride;        // the longest chain the launch may meet
    const int kpm = kpm_for(ncols);
    if (kpm < 0) return PE_ERR_SIZE;
    if (kpm > NARROW && precision != PE_PRECISION_F64) return PE_ERR_SIZE;   // mixed form: up to 32 columns
    if (warp_mode && (kpm > WMAXN || split || precision == PE_PRECISION_COMPENSATED)) return PE_ERR_SIZE;
    if (tpl == 0) {
        tpl = warp_mode ? 2 : default_tpl(kpm, precision);     // warp form: two-thread lanes (8 columns: three CTAs per SM)
        if (!warp_mode && !find_chain_kernel(precision, tpl, kpm)) tpl = find_chain_kernel(precision, 2, kpm) ? 2 : 4;
    }
    if (tpl_index(tpl) < 0) return PE_ERR_ARG;
    void* fn = warp_mode ? find_warp_kernel(precision, tpl, kpm) : find_chain_kernel(precision, tpl, kpm);
    if (!fn) return PE_ERR_SIZE;
    const int bmax = max_block(fn);
    if (bmax < 32) return PE_ERR_CUDA;
    // default CTA: 128 threads (as many warps per SM as 256-thread CTAs, twice the CTAs to overlap the
    // per-step serial phases of one stream with the sweeps of others)
    // warp form: one stream per warp, block_threads / 32 streams per CTA (default 8)
    const int block = warp_mode ? (block_threads ? block_threads : 32 * WARPS)
                                : (block_threads ? block_threads : (bmax < 128 ? bmax : 128));
    if (block < 32 || block > 256 || block > bmax || (block & 31)) return PE_ERR_ARG;
    if (!warp_mode && block < ncols) return PE_ERR_ARG;
    const size_t smem_fix = smem_fixed_bytes_for(kpm, precision);
    const size_t smem = warp_mode ? warp_smem_bytes(precision, tpl, kpm, block / 32)
                                  : smem_fix + (size_t)m_max * sizeof(double);
    const int cap = max_smem_optin();
    if (cap <= 0) return PE_ERR_CUDA;
    if (smem > (size_t)cap) return PE_ERR_SIZE;
    cudaStream_t st = (cudaStream_t)stream;
    PE_CUDA_TRY(cudaMemsetAsync(d_workspace, 0, zero_status ? WS_BYTES : sizeof(unsigned long long), st));
    if (S == 0) return PE_OK;
    const int klast = (k_last > 0 && k_last < n_stride) ? k_last : n_stride;
    int per_sm = 0;
    int rc = launch_prepare(fn, block, smem, &per_sm);
    if (rc != PE_OK) return rc;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int64_t grid = grid_ctas > 0 ? grid_ctas : (int64_t)sms * per_sm;
    const int64_t units = warp_mode ? (S + block / 32 - 1) / (block / 32) : S;   // streams in flight per CTA
    if (grid > units) grid = units;
    if (grid < 1) grid = 1;
    ChainParams p;
    p.acol = (const double2*)d_acol;
    p.inst_off = d_inst_off; p.inst_m = d_inst_m; p.inst_n = d_inst_n; p.G = G;
    p.S = S; p.dp = d_dp; p.nk = d_nk; p.cols = d_cols; p.n_stride = n_stride;
    p.uniforms = d_uniforms; p.seeds = d_seeds; p.seed_row = d_seed_row; p.rng_off = d_rng_off; p.order = d_order;
    p.qrange = d_qrange;
    p.rows = d_rows; p.occ = d_occ; p.occ_stride = d_occ ? occ_stride : m_max; p.marg = d_marg; p.marg_stride = marg_stride;
    p.queue = (unsigned long long*)d_workspace;
    p.status = (int*)((char*)d_workspace + 8);
    p.detail = (long long*)((char*)d_workspace + 16);
    p.m_cap = m_max;
    // Guard bands of the mixed forms.  Mixed: the largest CDF deviation from FP64 measured on chain rows of
    // Haar circuits (m = 400, 784, 900; 24-64 chains, up to 32 columns) is 1.1e-6 at 20 columns and grows
    // about 1.19x per column (7.8e-6 at 32); the band is 8x that envelope, about 2 tau m of the draws
    // redo their step in FP64.  Compensated: its blocks are FP64-accurate (~1e-10); the band only keeps
    // its picks the FP64 form's where the two round differently.
    p.tau = precision == PE_PRECISION_COMPENSATED ? 1.0e-8 : 8.0e-6;
    p.tau_log2g = 0.251;       // log2(1.19)
    p.k_first = k_first;
    p.k_stop = split ? (k_split - 1 < klast ? k_split - 1 : klast) : (k_last > 0 ? klast : 0);
    p.split_cap = (split && d_qrange) ? nq : -1;
    void* args[] = {&p};
    PE_CUDA_TRY(cudaLaunchKernel(fn, dim3((unsigned)grid), dim3(block), args, smem, st));
    if (!split) return PE_OK;
    // the mixed form's guard band: flagged streams redo the step with the FP64 kernels (second pass)
    const int npass = precision != PE_PRECISION_F64 ? 2 : 1;
    void* fpart[2] = {find_split_partial_kernel(precision, tpl, kpm), find_split_partial_kernel(PE_PRECISION_F64, tpl, kpm)};
    void* fdraw[2] = {find_split_draw_kernel(precision, tpl, kpm), find_split_draw_kernel(PE_PRECISION_F64, tpl, kpm)};
    int64_t gpart[2], gdraw[2];
    const int64_t items = nq * (int64_t)nch;
    for (int q = 0; q < npass; ++q) {
        if (!fpart[q] || !fdraw[q]) return PE_ERR_SIZE;
        int per_part = 0, per_draw = 0;
        const int pq = q == 0 ? precision : PE_PRECISION_F64;
        const size_t sdraw = smem_fixed_bytes_for(kpm, pq) + (size_t)m_max * sizeof(double);
        if ((rc = launch_prepare(fpart[q], block, smem_fixed_bytes_for(kpm, pq), &per_part)) != PE_OK) return rc;
        if ((rc = launch_prepare(fdraw[q], block, sdraw, &per_draw)) != PE_OK) return rc;
        gpart[q] = items < (int64_t)sms * per_part ? items : (int64_t)sms * per_part;
        gdraw[q] = nq < (int64_t)sms * per_draw ? nq : (int64_t)sms * per_draw;
    }
    SplitParams sp;
    sp.c = p;
    sp.nch = nch;
    sp.nq = nq;
    sp.partial = (double2*)((char*)d_workspace + WS_BYTES);
    sp.flag = (int*)((char*)d_workspace + WS_BYTES + part_bytes);
    void* sargs[] = {&sp};
    const int ksplit_last = (nk_max > 0 && nk_max < klast) ? nk_max : klast;
    for (int k = (k_split > k_first ? k_split : k_first); k <= ksplit_last; ++k) {
        sp.k = k;
        for (int q = 0; q < npass; ++q) {
            sp.pass = q;
            const int pq = q == 0 ? precision : PE_PRECISION_F64;
            PE_CUDA_TRY(cudaLaunchKernel(fpart[q], dim3((unsigned)gpart[q]), dim3(block), sargs,
                                         smem_fixed_bytes_for(kpm, pq), st));
            PE_CUDA_TRY(cudaLaunchKernel(fdraw[q], dim3((unsigned)gdraw[q]), dim3(block), sargs,
                                         smem_fixed_bytes_for(kpm, pq) + (size_t)m_max * sizeof(double), st));
        }
    }
    return PE_OK;
}

extern "C" int pe_fock_chain(int precision, const double* d_acol, const int64_t* d_inst_off, const int32_t* d_inst_m,
                             const int32_t* d_inst_n, int G, int m_max, int64_t S, const int64_t* d_dp,
                             const int32_t* d_nk, const int64_t* d_cols, int n_stride, const double* d_uniforms,
                             const int64_t* d_seeds, const int64_t* d_seed_row, const int64_t* d_rng_off,
                             const int64_t* d_order, int64_t* d_rows, int64_t* d_occ, int occ_stride, double* d_marg,
                             int marg_stride, void* d_workspace, size_t workspace_bytes, int block_threads, int tpl,
                             int grid_ctas, void* stream) {
    return chain_launch(precision, d_acol, d_inst_off, d_inst_m, d_inst_n, G, m_max, S, d_dp, d_nk, d_cols, n_stride,
                        d_uniforms, d_seeds, d_seed_row, d_rng_off, d_order, d_rows, d_occ, occ_stride, d_marg,
                        marg_stride, d_workspace, workspace_bytes, block_threads, tpl, grid_ctas, 0, 1, stream);
}

extern "C" int pe_fock_chain_range(int precision, const double* d_acol, const int64_t* d_inst_off,
                                   const int32_t* d_inst_m, const int32_t* d_inst_n, int G, int m_max, int64_t S,
                                   const int64_t* d_dp, const int32_t* d_nk, const int64_t* d_cols, int n_stride,
                                   const double* d_uniforms, const int64_t* d_seeds, const int64_t* d_seed_row,
                                   const int64_t* d_rng_off, const int64_t* d_order, int64_t* d_rows, int64_t* d_occ,
                                   int occ_stride, double* d_marg, int marg_stride, void* d_workspace,
                                   size_t workspace_bytes, int block_threads, int tpl, int grid_ctas,
                                   const int64_t* d_qrange, int nk_max, int warp, void* stream) {
    if (!d_qrange || !d_order || !d_nk || nk_max < 1 || (warp != 0 && warp != 1)) return PE_ERR_ARG;
    return chain_launch(precision, d_acol, d_inst_off, d_inst_m, d_inst_n, G, m_max, S, d_dp, d_nk, d_cols, n_stride,
                        d_uniforms, d_seeds, d_seed_row, d_rng_off, d_order, d_rows, d_occ, occ_stride, d_marg,
                        marg_stride, d_workspace, workspace_bytes, block_threads, tpl, grid_ctas, 0, 1,
                        stream, warp == 1, 1, 0, true, d_qrange, nk_max);
}

extern "C" size_t pe_range_split_workspace_bytes(int64_t split_slots, int nch) {
    const size_t q = (size_t)(split_slots < 0 ? 0 : split_slots);
    return WS_BYTES + q * (size_t)(nch < 1 ? 1 : nch) * MAXN * sizeof(double2) + q * sizeof(int);
}

extern "C" int pe_fock_chain_range_split(int precision, const double* d_acol, const int64_t* d_inst_off,
                                         const int32_t* d_inst_m, const int32_t* d_inst_n, int G, int m_max,
                                         int64_t S, const int64_t* d_dp, const int32_t* d_nk, const int64_t* d_cols,
                                         int n_stride, const double* d_uniforms, const int64_t* d_seeds,
                                         const int64_t* d_seed_row, const int64_t* d_rng_off, const int64_t* d_order,
                                         int64_t* d_rows, int64_t* d_occ, int occ_stride, double* d_marg,
                                         int marg_stride, void* d_workspace, size_t workspace_bytes,
                                         int block_threads, int tpl, const int64_t* d_qrange, int nk_max,
                                         int k_split, int nch, int64_t split_slots, void* stream) {
    if (!d_qrange || !d_order || !d_nk || nk_max < 1 || k_split < 2 || nch < 1 || split_slots < 1) return PE_ERR_ARG;
    return chain_launch(precision, d_acol, d_inst_off, d_inst_m, d_inst_n, G, m_max, S, d_dp, d_nk, d_cols, n_stride,
                        d_uniforms, d_seeds, d_seed_row, d_rng_off, d_order, d_rows, d_occ, occ_stride, d_marg,
                        marg_stride, d_workspace, workspace_bytes, block_threads, tpl, 0, k_split, nch, stream, false,
                        1, 0, true, d_qrange, nk_max, split_slots);
}

extern "C" int pe_fock_chain_warp(int precision, const double* d_acol, const int64_t* d_inst_off,
                                  const int32_t* d_inst_m, const int32_t* d_inst_n, int G, int m_max, int64_t S,
                                  const int64_t* d_dp, const int32_t* d_nk, const int64_t* d_cols, int n_stride,
                                  const double* d_uniforms, const int64_t* d_seeds, const int64_t* d_seed_row,
                                  const int64_t* d_rng_off, const int64_t* d_order, int64_t* d_rows, int64_t* d_occ,
                                  int occ_stride, double* d_marg, int marg_stride, void* d_workspace,
                                  size_t workspace_bytes, int tpl, int grid_ctas, void* stream) {
    return chain_launch(precision, d_acol, d_inst_off, d_inst_m, d_inst_n, G, m_max, S, d_dp, d_nk, d_cols, n_stride,
                        d_uniforms, d_seeds, d_seed_row, d_rng_off, d_order, d_rows, d_occ, occ_stride, d_marg,
                        marg_stride, d_workspace, workspace_bytes, 0, tpl, grid_ctas, 0, 1, stream, true);
}

extern "C" size_t pe_chain_split_workspace_bytes(int64_t S, int nch) {
    const size_t s = (size_t)(S < 0 ? 0 : S);
    return WS_BYTES + s * (size_t)(nch < 1 ? 1 : nch) * MAXN * sizeof(double2) + s * sizeof(int);
}

extern "C" int pe_fock_chain_split(int precision, const double* d_acol, const int64_t* d_inst_off,
                                   const int32_t* d_inst_m, const int32_t* d_inst_n, int G, int m_max, int64_t S,
                                   const int64_t* d_dp, const int32_t* d_nk, const int64_t* d_cols, int n_stride,
                                   const double* d_uniforms, const int64_t* d_seeds, const int64_t* d_seed_row,
                                   const int64_t* d_rng_off, const int64_t* d_order, int64_t* d_rows, int64_t* d_occ,
                                   int occ_stride, double* d_marg, int marg_stride, int k_split, int nch,
                                   void* d_workspace, size_t workspace_bytes, int block_threads, int tpl, void* stream) {
    if (k_split < 2 || nch < 1) return PE_ERR_ARG;
    return chain_launch(precision, d_acol, d_inst_off, d_inst_m, d_inst_n, G, m_max, S, d_dp, d_nk, d_cols, n_stride,
                        d_uniforms, d_seeds, d_seed_row, d_rng_off, d_order, d_rows, d_occ, occ_stride, d_marg,
                        marg_stride, d_workspace, workspace_bytes, block_threads, tpl, 0, k_split, nch, stream);
}

extern "C" size_t pe_adaptive_workspace_bytes(int64_t S, int nch) {
    const size_t s = (size_t)(S < 0 ? 0 : S);
    return align16(WS_BYTES + split_bytes(S < 0 ? 0 : S, nch)) + align16(s * sizeof(int32_t)) + 2 * s * sizeof(int64_t);
}

extern "C" int pe_fock_chain_adaptive(int precision, const double* d_acol, const int64_t* d_inst_off,
                                      const int32_t* d_inst_m, const int32_t* d_inst_n, int G, int m_max, int64_t S,
                                      const int64_t* d_dp, const int64_t* d_cols, int n_stride,
                                      const double* d_uniforms, const int64_t* d_seeds, const int64_t* d_seed_row,
                                      const int64_t* d_rng_off, int64_t* d_rows, int n_prefix,
                                      const uint8_t* d_avoid, uint8_t* d_alive, int64_t* d_occ, int occ_stride,
                                      int k_split, int nch, void* d_workspace, size_t workspace_bytes,
                                      int block_threads, int tpl, int mode, void* stream) {
    if (n_prefix < 0 || n_prefix > n_stride || (mode != 0 && mode != 1)) return PE_ERR_ARG;
    if (k_split < 0 || (k_split > 0 && (k_split < 2 || nch < 1))) return PE_ERR_ARG;
    if (mode == 1 && k_split > 0) return PE_ERR_ARG;
    if (d_avoid && !d_alive) return PE_ERR_ARG;
    if (!d_rows || !d_workspace || S < 0) return PE_ERR_ARG;
    const int ks = (k_split > 0 && k_split <= n_stride) ? k_split : 0;
    const bool warp = mode == 1;
    if (!d_avoid || n_prefix == n_stride) {
        if (d_alive && S > 0) PE_CUDA_TRY(cudaMemsetAsync(d_alive, 1, (size_t)S, (cudaStream_t)stream));
        return chain_launch(precision, d_acol, d_inst_off, d_inst_m, d_inst_n, G, m_max, S, d_dp, nullptr, d_cols,
                            n_stride, d_uniforms, d_seeds, d_seed_row, d_rng_off, nullptr, d_rows, d_occ, occ_stride,
                            nullptr, m_max, d_workspace, workspace_bytes, block_threads, tpl, 0, ks, nch, stream, warp,
                            n_prefix + 1, 0, true);
    }
    if (workspace_bytes < pe_adaptive_workspace_bytes(S, ks ? nch : 0) || ((uintptr_t)d_workspace & 15u))
        return PE_ERR_SIZE;
    if (d_occ && occ_stride < m_max) return PE_ERR_ARG;
    char* w = (char*)d_workspace;
    const size_t o_nk = align16(WS_BYTES + split_bytes(S, ks ? nch : 0));
    AvoidParams a;
    a.rows = d_rows; a.n_stride = n_stride; a.avoid = d_avoid; a.m_max = m_max; a.alive = d_alive;
    a.nk = (int32_t*)(w + o_nk);
    a.rng = (int64_t*)(w + o_nk + align16((size_t)S * sizeof(int32_t)));
    a.scan = a.rng + S;
    a.off0 = d_rng_off; a.S = S; a.n = n_stride; a.occ = d_occ; a.occ_stride = occ_stride;
    a.status = (int*)(w + 8);
    a.detail = (long long*)(w + 16);
    cudaStream_t st = (cudaStream_t)stream;
    PE_CUDA_TRY(cudaMemsetAsync(d_workspace, 0, WS_BYTES, st));
    if (S == 0) return PE_OK;
    for (int k = n_prefix + 1; k <= n_stride; ++k) {
        a.col = k == n_prefix + 1 ? -1 : k - 2;            // no check before the first free step
        a.zero_dead = 0;
        avoid_update_kernel<<<1, 1024, 0, st>>>(a);
        PE_CUDA_TRY(cudaGetLastError());
        const int rc = chain_launch(precision, d_acol, d_inst_off, d_inst_m, d_inst_n, G, m_max, S, d_dp, a.nk,
                                    d_cols, n_stride, d_uniforms, d_seeds, d_seed_row, a.rng, nullptr, d_rows,
                                    k == n_stride ? d_occ : nullptr, occ_stride, nullptr, m_max, d_workspace,
                                    workspace_bytes, block_threads, tpl, 0, ks, nch, stream, warp, k, k, false);
        if (rc != PE_OK) return rc;
    }
    a.col = n_stride - 1;                                 // the last photon is checked too
    a.zero_dead = 1;
    avoid_update_kernel<<<1, 1024, 0, st>>>(a);
    return ::pe::launch_status();
}

extern "C" int pe_cofactors_rows(int precision, const double* d_a, const int64_t* d_rows, int64_t S, int m, int K,
                                 double* d_p, void* d_workspace, size_t workspace_bytes, int block_threads, int tpl,
                                 void* stream) {
    if (!prec_ok(precision)) return PE_ERR_ARG;
    if (S < 0 || m < 1 || K < 1 || !d_a || !d_p || !d_workspace) return PE_ERR_ARG;
    if (K > 1 && !d_rows) return PE_ERR_ARG;
    if (workspace_bytes < WS_BYTES || ((uintptr_t)d_workspace & 15u)) return PE_ERR_SIZE;
    const int kpm = kpm_for(K);
    if (kpm < 0) return PE_ERR_SIZE;
    if (kpm > NARROW && precision != PE_PRECISION_F64) return PE_ERR_SIZE;
    if (tpl == 0) tpl = precision == PE_PRECISION_COMPENSATED ? default_tpl(kpm, precision) : (kpm <= 8 ? 1 : (kpm <= 40 ? 2 : 4));
    if (tpl_index(tpl) < 0) return PE_ERR_ARG;
    void* fn = find_cofactor_kernel(precision, tpl, kpm);
    if (!fn) return PE_ERR_SIZE;
    const int bmax = max_block(fn);
    if (bmax < 32) return PE_ERR_CUDA;
    const int block = block_threads ? block_threads : (bmax < 256 ? bmax : 256);
    if (block < 32 || block > 256 || block > bmax || (block & 31) || block < K) return PE_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    PE_CUDA_TRY(cudaMemsetAsync(d_workspace, 0, WS_BYTES, st));
    if (S == 0) return PE_OK;
    const size_t smem = smem_fixed_bytes_for(kpm, precision);
    int per_sm = 0;
    int rc = launch_prepare(fn, block, smem, &per_sm);
    if (rc != PE_OK) return rc;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int64_t grid = (int64_t)sms * per_sm;
    if (grid > S) grid = S;
    const double2* a = (const double2*)d_a;
    double2* pp = (double2*)d_p;
    int* status = (int*)((char*)d_workspace + 8);
    long long* detail = (long long*)((char*)d_workspace + 16);
    void* args[] = {(void*)&a, (void*)&d_rows, (void*)&S, (void*)&m, (void*)&K, (void*)&pp, (void*)&status, (void*)&detail};
    PE_CUDA_TRY(cudaLaunchKernel(fn, dim3((unsigned)grid), dim3(block), args, smem, st));
    return PE_OK;
}

extern "C" int pe_split_slots(int precision, int n_stride, int block_threads, int tpl) {
    if (!prec_ok(precision)) return PE_ERR_ARG;
    const int kpm = kpm_for(n_stride);
    if (n_stride < 1 || kpm < 0) return PE_ERR_SIZE;
    if (kpm > NARROW && precision != PE_PRECISION_F64) return PE_ERR_SIZE;
    if (tpl == 0) {
        tpl = default_tpl(kpm, precision);
        if (!find_chain_kernel(precision, tpl, kpm)) tpl = find_chain_kernel(precision, 2, kpm) ? 2 : 4;
    }
    if (tpl_index(tpl) < 0) return PE_ERR_ARG;
    void* fn = find_split_partial_kernel(precision, tpl, kpm);
    if (!fn) return PE_ERR_SIZE;
    const int bmax = max_block(fn);
    if (bmax < 32) return PE_ERR_CUDA;
    const int block = block_threads ? block_threads : (bmax < 128 ? bmax : 128);
    if (block < 32 || block > 256 || block > bmax || (block & 31)) return PE_ERR_ARG;
    int per_sm = 0, dev = 0, sms = 0;
    const int rc = launch_prepare(fn, block, smem_fixed_bytes_for(kpm, precision), &per_sm);
    if (rc != PE_OK) return rc;
    PE_CUDA_TRY(cudaGetDevice(&dev));
    PE_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    return sms * per_sm;
}

extern "C" int pe_pipe_probe(int precision, int iters, void* d_out, size_t out_bytes, double* flops, void* stream) {
    if ((precision != PE_PRECISION_F64 && precision != PE_PRECISION_MIXED) || iters < 1 || !d_out || !flops)
        return PE_ERR_ARG;
    int dev = 0, sms = 0;
    PE_CUDA_TRY(cudaGetDevice(&dev));
    PE_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int threads = 256, blocks = sms * 8;
    const size_t need = (size_t)blocks * threads * (precision == PE_PRECISION_F64 ? 8 : 4);
    if (out_bytes < need) return PE_ERR_SIZE;
    cudaStream_t st = (cudaStream_t)stream;
    if (precision == PE_PRECISION_F64)
        pipe_probe_kernel<double><<<blocks, threads, 0, st>>>((double*)d_out, 0.999999, 1e-7, iters);
    else
        pipe_probe_kernel<float><<<blocks, threads, 0, st>>>((float*)d_out, 0.999999f, 1e-7f, iters);
    PE_CUDA_TRY(cudaGetLastError());
    *flops = 2.0 * 8.0 * (double)iters * (double)blocks * (double)threads;
    return PE_OK;
}

// ---------------------------------------------------------------------------------------- allocation-free chain
// For callers that cannot allocate device memory themselves at the time they sample: code running in a
// host callback or another context where CUDA allocation calls are not allowed, a serving process whose
// device memory is all handed out by its own arena, or a foreign-language binding that can pass the
// buffers it was given but has no way to call cudaMalloc.  pe_fock_chain needs a small caller-provided
// workspace (the work-queue counter and the status word); this entry point keeps that scratch in a
// static device array instead, so the caller passes inputs and outputs only.
//
// The array is PE_NOALLOC_SCRATCH_BYTES long; every GPU that loads this library holds it until the
// process exits.  All calls share it and it keeps the last call's contents: each call clears the part
// that must start at zero (queue counter, status word) on its stream before launching, and calls whose
// kernels overlap on the GPU (different streams, or different host threads on one device) race on it.
constexpr size_t PE_NOALLOC_SCRATCH_BYTES = 4096;
static_assert(WS_BYTES <= PE_NOALLOC_SCRATCH_BYTES, "the chain workspace must fit the static scratch");
static __device__ __align__(256) unsigned char g_noalloc_scratch[PE_NOALLOC_SCRATCH_BYTES];

constexpr int PE_NOALLOC_MAX_DEVICES = 64;
static void* g_noalloc_ptr[PE_NOALLOC_MAX_DEVICES];
static std::mutex g_noalloc_mutex;

// Device address of the scratch on the current device.  The host-side name of the array is only a
// stand-in; the address comes from cudaGetSymbolAddress, once per device, with that device current.
static int noalloc_scratch(void** out) {
    int dev = 0;
    PE_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= PE_NOALLOC_MAX_DEVICES) return PE_ERR_SIZE;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return PE_ERR_CUDA;
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return PE_OK;
}

extern "C" int pe_fock_chain_noalloc(int precision, const double* d_acol, const int64_t* d_inst_off,
                                     const int32_t* d_inst_m, const int32_t* d_inst_n, int G, int m_max, int64_t S,
                                     const int64_t* d_dp, const int32_t* d_nk, const int64_t* d_cols, int n_stride,
                                     const double* d_uniforms, const int64_t* d_seeds, const int64_t* d_seed_row,
                                     const int64_t* d_rng_off, const int64_t* d_order, int64_t* d_rows, int64_t* d_occ,
                                     int occ_stride, double* d_marg, int marg_stride, int* d_status,
                                     int block_threads, int tpl, int grid_ctas, void* stream) {
    if (pe_chain_workspace_bytes(S) > PE_NOALLOC_SCRATCH_BYTES) return PE_ERR_SIZE;
    void* scratch = nullptr;
    const int rc0 = noalloc_scratch(&scratch);
    if (rc0 != PE_OK) return rc0;
    const int rc = pe_fock_chain(precision, d_acol, d_inst_off, d_inst_m, d_inst_n, G, m_max, S, d_dp, d_nk, d_cols,
                                 n_stride, d_uniforms, d_seeds, d_seed_row, d_rng_off, d_order, d_rows, d_occ,
                                 occ_stride, d_marg, marg_stride, scratch, PE_NOALLOC_SCRATCH_BYTES, block_threads, tpl,
                                 grid_ctas, stream);
    if (rc != PE_OK) return rc;
    if (d_status)
        PE_CUDA_TRY(cudaMemcpyAsync(d_status, (const char*)scratch + 8, sizeof(int), cudaMemcpyDeviceToDevice,
                                    (cudaStream_t)stream));
    return PE_OK;
}
