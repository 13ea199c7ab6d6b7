// INT8 tensor-core (tcgen05, kind::i8) self-test and throughput probe:
// C[128 x N] = A[128 x K] * B[N x K]^T with int32 accumulation in TMEM.
// Every CTA of the grid computes the same product from its own shared-memory
// copy (only CTA 0 writes C), so `grid` CTAs x `reps` passes measure the
// sustained MMA rate; the test compares C against an integer reference.
#include <cuda_runtime.h>
#include <stdint.h>

#include "e8qc.h"
#include "internal.h"
#include "tc.cuh"
#include "tma.cuh"

namespace e8qc {
bool is_device_ptr(const void* p);
void set_last_error(const std::string& s);

namespace {

__global__ void __launch_bounds__(128) tc_i8_gemm_kernel(const int8_t* __restrict__ A, const int8_t* __restrict__ B,
                                                         int N, int K, int reps, int32_t* __restrict__ C,
                                                         uint32_t* __restrict__ err) {
    extern __shared__ __align__(128) unsigned char sm[];
    __shared__ uint32_t s_tmem;
    __shared__ __align__(8) uint64_t s_bar;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    unsigned char* sa = sm;                        // 128 x K interleaved
    unsigned char* sb = sm + 128 * K;              // N x K interleaved
    for (int e = tid; e < 128 * K; e += 128) {
        const int r = e / K, k = e - r * K;
        sa[tc::il_offset(r, k, K)] = static_cast<unsigned char>(A[e]);
    }
    for (int e = tid; e < N * K; e += 128) {
        const int r = e / K, k = e - r * K;
        sb[tc::il_offset(r, k, K)] = static_cast<unsigned char>(B[e]);
    }
    uint32_t ncols = 32;
    while (ncols < static_cast<uint32_t>(N)) ncols <<= 1;
    if (warp == 0) {
        tc::tmem_alloc(&s_tmem, ncols);
        tc::tmem_relinquish();
    }
    if (tid == 0) {
        mbar_init(&s_bar, 1);
        fence_barrier_init();
    }
    tc::fence_smem_to_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = s_tmem;
    if (tid == 0) {
        const uint32_t idesc = tc::idesc_i8(128, N);
        const uint32_t sbo = static_cast<uint32_t>(K / 16) * 128u;
        const uint32_t a0 = tc::saddr(sa), b0 = tc::saddr(sb);
        for (int rep = 0; rep < reps; ++rep) {
            for (int ks = 0; ks < K / 32; ++ks) {
                const uint64_t ad = tc::smem_desc(a0 + 256u * ks, 128u, sbo);
                const uint64_t bd = tc::smem_desc(b0 + 256u * ks, 128u, sbo);
                tc::mma_i8(tmem, ad, bd, idesc, (rep > 0 || ks > 0) ? 1u : 0u);
            }
        }
        tc::mma_commit(&s_bar);
    }
    const bool got = mbar_wait_bounded(&s_bar, 0);
    if (!got && lane == 0) atomicOr(err, kErrWaitTimeout);
    tc::fence_after_sync();
    if (got && blockIdx.x == 0) {
        for (int c0 = 0; c0 < N; c0 += 8) {
            uint32_t r[8];
            tc::tmem_ld8(tmem + ((static_cast<uint32_t>(warp) * 32u) << 16) + static_cast<uint32_t>(c0), r);
            tc::tmem_ld_wait();
            for (int j = 0; j < 8; ++j) C[(warp * 32 + lane) * N + c0 + j] = static_cast<int32_t>(r[j]);
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, ncols);
}

}  // namespace
}  // namespace e8qc

using namespace e8qc;

extern "C" int e8qc_tc_i8_gemm(int device, const int8_t* A, const int8_t* B, int n, int k, int reps, int grid,
                               int32_t* C, float* ms) {
    try {
        if (n < 16 || n > 256 || n % 16 != 0) fail(E8QC_EINVAL, "n must be a multiple of 16 in [16, 256]");
        if (k < 32 || k > 256 || k % 32 != 0) fail(E8QC_EINVAL, "k must be a multiple of 32 in [32, 256]");
        if (reps < 1 || grid < 1 || grid > 4096) fail(E8QC_EINVAL, "reps and grid must be positive");
        if (!A || !B || !C) fail(E8QC_EINVAL, "null buffer");
        int prev = 0;
        E8QC_CUDA(cudaGetDevice(&prev));
        E8QC_CUDA(cudaSetDevice(device));
        struct Restore {
            int d;
            ~Restore() { cudaSetDevice(d); }
        } restore{prev};
        const size_t abytes = 128u * static_cast<size_t>(k), bbytes = static_cast<size_t>(n) * k,
                     cbytes = 128u * static_cast<size_t>(n) * 4;
        void *da = nullptr, *db = nullptr, *dc = nullptr, *de = nullptr;
        E8QC_CUDA(cudaMalloc(&da, abytes));
        E8QC_CUDA(cudaMalloc(&db, bbytes));
        E8QC_CUDA(cudaMalloc(&dc, cbytes));
        E8QC_CUDA(cudaMalloc(&de, 4));
        struct Free {
            void *a, *b, *c, *e;
            ~Free() {
                cudaFree(a);
                cudaFree(b);
                cudaFree(c);
                cudaFree(e);
            }
        } fr{da, db, dc, de};
        E8QC_CUDA(cudaMemcpy(da, A, abytes, is_device_ptr(A) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice));
        E8QC_CUDA(cudaMemcpy(db, B, bbytes, is_device_ptr(B) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice));
        E8QC_CUDA(cudaMemset(de, 0, 4));
        const size_t smem = abytes + bbytes;
        E8QC_CUDA(cudaFuncSetAttribute(tc_i8_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem)));
        cudaEvent_t e0, e1;
        E8QC_CUDA(cudaEventCreate(&e0));
        E8QC_CUDA(cudaEventCreate(&e1));
        E8QC_CUDA(cudaEventRecord(e0));
        tc_i8_gemm_kernel<<<grid, 128, smem>>>(static_cast<const int8_t*>(da), static_cast<const int8_t*>(db), n, k,
                                              reps, static_cast<int32_t*>(dc), static_cast<uint32_t*>(de));
        E8QC_CUDA(cudaGetLastError());
        E8QC_CUDA(cudaEventRecord(e1));
        E8QC_CUDA(cudaEventSynchronize(e1));
        float t = 0.0f;
        E8QC_CUDA(cudaEventElapsedTime(&t, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        uint32_t err = 0;
        E8QC_CUDA(cudaMemcpy(&err, de, 4, cudaMemcpyDeviceToHost));
        if (err) fail(E8QC_ETIMEOUT, "MMA completion wait gave up");
        E8QC_CUDA(cudaMemcpy(C, dc, cbytes, is_device_ptr(C) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost));
        if (ms) *ms = t;
        return E8QC_OK;
    } catch (const Error& e) {
        set_last_error(e.msg);
        return e.code;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return E8QC_EINVAL;
    }
}
