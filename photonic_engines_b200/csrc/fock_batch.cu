// Device-side partition of lossy / partially distinguishable shots into chains, for the batched
// sampler (many instances, one persistent chain launch, CUDA-graph replay).  The law is the
// reference's shared imperfections model (photonic_engines/imperfections.py:465-590): every input
// photon is lost with probability 1 - eta; a surviving one interferes with probability x (x-model)
// and is otherwise alone in its own internal mode.  The interfering photons of a shot form one chain
// in a uniformly random order (sigma); each lone photon is a one-photon chain, whose draw
// |U[rho, col]|^2 is the reference's classical routing (imperfections.py:576-590).  The draws come
// from Philox4x32-10 keyed by a device-resident key, so the partition is graph-capturable; they are
// not the reference's host draws (the drop-in `fock_sample` keeps those), the law is the same.
#include <cuda_runtime.h>
#include <stdint.h>

#include "pe_b200.h"
#include "pe_device.cuh"
#include "pe_errors.h"

namespace pe {

// Uniform in [0, 1) with 53 random bits from two Philox words of counter 2c, 2c + 1.
static __device__ __forceinline__ double u01(uint64_t key, uint32_t c) {
    const uint32_t a = philox_word0(key, 2u * c) >> 5, b = philox_word0(key, 2u * c + 1u) >> 6;
    return ((double)a * 67108864.0 + (double)b) * (1.0 / 9007199254740992.0);
}

// One thread per shot.  Slot layout per shot: slot 0 is the interfering chain, slots 1..n_stride the
// lone photons (when `singles`); chain c = s * slots + q, out_row[c] = s.
__global__ void partition_kernel(const int64_t* __restrict__ dp, const int32_t* __restrict__ inst_n,
                                 const double* __restrict__ eta, const double* __restrict__ x, int64_t S, int n_stride,
                                 int singles, const int64_t* __restrict__ key_ptr, int64_t* __restrict__ cols,
                                 int32_t* __restrict__ nk, int64_t* __restrict__ chain_dp, int64_t* __restrict__ out_row,
                                 int* __restrict__ status) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) return;
    const int slots = singles ? 1 + n_stride : 1;
    const int64_t g = dp[s];
    const int n = inst_n[g];
    const uint64_t key = (uint64_t)key_ptr[0];
    const double e = eta[g], xx = x[g];
    if (n < 0 || n > n_stride || n > MAXN) {
        atomicCAS(status, 0, PE_ERR_DEVICE);
        for (int q = 0; q < slots; ++q) { nk[s * slots + q] = 0; chain_dp[s * slots + q] = g; out_row[s * slots + q] = s; }
        return;
    }
    int good[MAXN];
    double sortkey[MAXN];
    int ng = 0;
    for (int j = 0; j < n; ++j) {
        const uint32_t base = (uint32_t)((s * n_stride + j) * 3);
        const bool kept = u01(key, base) < e;
        const bool inter = kept && (xx >= 1.0 || u01(key, base + 1) < xx);
        int64_t* slot_cols = cols + (s * slots + 1 + j) * n_stride;
        if (singles) {
            const int64_t c = s * slots + 1 + j;
            nk[c] = (kept && !inter) ? 1 : 0;
            slot_cols[0] = j;
            chain_dp[c] = g;
            out_row[c] = s;
        }
        if (inter) {                                     // insertion by a uniform key: sigma uniform
            const double r = u01(key, base + 2);
            int i = ng++;
            while (i > 0 && sortkey[i - 1] > r) { sortkey[i] = sortkey[i - 1]; good[i] = good[i - 1]; --i; }
            sortkey[i] = r;
            good[i] = j;
        }
    }
    if (singles) for (int j = n; j < n_stride; ++j) {
        const int64_t c = s * slots + 1 + j;
        nk[c] = 0;
        cols[c * n_stride] = 0;
        chain_dp[c] = g;
        out_row[c] = s;
    }
    const int64_t c0 = s * slots;
    for (int i = 0; i < n_stride; ++i) cols[c0 * n_stride + i] = i < ng ? good[i] : 0;
    nk[c0] = ng;
    chain_dp[c0] = g;
    out_row[c0] = s;
}

// Occupations of the shots from the chains' ordered rows: occ[out_row[c], rows[c, j]] += 1, j < nk[c].
__global__ void scatter_occ_kernel(const int64_t* __restrict__ rows, const int32_t* __restrict__ nk,
                                   const int64_t* __restrict__ out_row, int64_t C, int n_stride, int64_t* __restrict__ occ,
                                   int occ_stride, int64_t S, int* __restrict__ status) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) return;
    const int64_t r = out_row[c];
    const int k = nk[c];
    if (r < 0 || r >= S || k < 0 || k > n_stride) { atomicCAS(status, 0, PE_ERR_DEVICE); return; }
    for (int j = 0; j < k; ++j) {
        const int64_t mode = rows[c * n_stride + j];
        if (mode < 0 || mode >= occ_stride) { atomicCAS(status, 0, PE_ERR_DEVICE); continue; }
        atomicAdd((unsigned long long*)&occ[r * occ_stride + mode], 1ull);
    }
}

}  // namespace pe

using namespace pe;

extern "C" int pe_partition_shots(const int64_t* d_dp, const int32_t* d_inst_n, const double* d_eta, const double* d_x,
                                  int64_t S, int n_stride, int singles, const int64_t* d_key, int64_t* d_cols,
                                  int32_t* d_nk, int64_t* d_chain_dp, int64_t* d_out_row, int* d_status, void* stream) {
    if (S < 0 || n_stride < 1 || n_stride > MAXN || !d_dp || !d_inst_n || !d_eta || !d_x || !d_key || !d_cols ||
        !d_nk || !d_chain_dp || !d_out_row || !d_status)
        return PE_ERR_ARG;
    if (S * (int64_t)n_stride * 3 >= (int64_t)1 << 31) return PE_ERR_SIZE;     // Philox counters stay 32-bit
    if (S == 0) return PE_OK;
    const int threads = 128;
    partition_kernel<<<(unsigned)((S + threads - 1) / threads), threads, 0, (cudaStream_t)stream>>>(
        d_dp, d_inst_n, d_eta, d_x, S, n_stride, singles, d_key, d_cols, d_nk, d_chain_dp, d_out_row, d_status);
    return ::pe::launch_status();
}

extern "C" int pe_scatter_occupations(const int64_t* d_rows, const int32_t* d_nk, const int64_t* d_out_row, int64_t C,
                                      int n_stride, int64_t* d_occ, int occ_stride, int64_t S, int* d_status,
                                      void* stream) {
    if (C < 0 || S < 0 || n_stride < 1 || occ_stride < 1 || !d_rows || !d_nk || !d_out_row || !d_occ || !d_status)
        return PE_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    PE_CUDA_TRY(cudaMemsetAsync(d_occ, 0, (size_t)S * occ_stride * sizeof(int64_t), st));
    if (C == 0) return PE_OK;
    const int threads = 128;
    scatter_occ_kernel<<<(unsigned)((C + threads - 1) / threads), threads, 0, st>>>(d_rows, d_nk, d_out_row, C, n_stride,
                                                                                   d_occ, occ_stride, S, d_status);
    return ::pe::launch_status();
}
