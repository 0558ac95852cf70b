// Blackwell (sm_100a) tensor-core GEMM for the learned preconditioner's
// channel mixing: C[M, N] = A[M, K] * B[N, K]^T, A and B BF16 row-major
// (both "K-major"), FP32 accumulation in tensor memory, with a fused epilogue
// functor that consumes the FP32 accumulators row by row.
//
// Data movement: TMA (cp.async.bulk.tensor.2d) loads 128-row tiles of A and
// the whole of B into shared memory with the 64-byte swizzle (one swizzle atom
// = 8 rows x 32 BF16 of K); one elected thread issues tcgen05.mma
// (kind::f16, M = 128, N = 32..256, K = 16 per instruction) into a TMEM
// accumulator of N columns, commits to an mbarrier, and the four warps read
// their 32 accumulator rows back with tcgen05.ld (32x32b shape: lane = row).
// The CTA is persistent over row tiles with an S-stage TMA pipeline on A, so
// the loads of the next tiles are in flight during the epilogue of this one.
//
// Every wait is bounded (about one second of device time); on a timeout the
// kernel records the error in *err, lets its own copies in flight land
// (again bounded), releases its tensor memory and returns.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <stdint.h>

namespace cg {
namespace umma {

constexpr int TILE_M = 128;
constexpr int KCHUNK = 32;                         // K elements per swizzle atom (64 bytes of BF16)
constexpr int A_CHUNK_BYTES = TILE_M * KCHUNK * 2;  // 8 KB per 128 x 32 chunk
constexpr unsigned long long WAIT_NS = 1000000000ull;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t *bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}
// Wait for the phase with the given parity to complete; false after ~1 s.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    if (mbar_try(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    for (;;) {
        if (mbar_try(bar, parity)) return true;
        if (global_ns() - t0 > WAIT_NS) return false;
    }
}

// 2-D tiled TMA load of box (x = inner coordinate in elements, y = row) into
// shared memory, completing `bar`'s transaction count.
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
            smem_u32(dst)),
        "l"((uint64_t)map), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor of a K-major operand tile stored with the
// 64-byte swizzle: rows of 64 bytes, 8-row groups 512 bytes apart (SBO), LBO
// unused for swizzled K-major layouts, version 1 (sm_100), layout type 4.
__device__ __forceinline__ uint64_t desc_k_sw64(uint32_t saddr) {
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)(512 >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)4 << 61;
    return d;
}

// Instruction descriptor: BF16 x BF16 -> FP32, both operands K-major, M = 128.
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(TILE_M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// 32 consecutive FP32 accumulator columns of this thread's row (lane).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// Shared memory of one CTA (bytes), for N output columns, KC chunks of 32 K,
// S pipeline stages on A.
__host__ __device__ constexpr size_t b_bytes(int n, int kc) { return (size_t)kc * n * 64; }
__host__ __device__ constexpr size_t round1k(size_t v) { return (v + 1023) & ~(size_t)1023; }
__host__ __device__ constexpr size_t smem_bytes(int n, int kc, int s) {
    return 1024 /* alignment slack */ + round1k(b_bytes(n, kc)) + (size_t)s * kc * A_CHUNK_BYTES + 256;
}
__host__ __device__ constexpr uint32_t tmem_cols(int n) { return n <= 32 ? 32u : n <= 64 ? 64u : n <= 128 ? 128u : 256u; }

// Epilogue interface: each thread works on its own copy of `epi`;
// e.row(row, acc_chunk, c0) is called for every valid row (< M) and every
// 32-column chunk c0 = 0, 32, ..., in order, then e.done(row).  The kernel
// returns at once while *gate != 0 (gate may be null).
template <int N, int KC, int S, class Epi>
__global__ void __launch_bounds__(128) k_gemm(const __grid_constant__ CUtensorMap ta,
                                              const __grid_constant__ CUtensorMap tb, long long M, Epi epi,
                                              int *err, const int *gate) {
    static_assert(N % 32 == 0 && N >= 32 && N <= 256, "N");
    if (gate && *(volatile const int *)gate) return;  // uniform for the whole grid
    Epi e = epi;
    extern __shared__ unsigned char smem_raw[];
    unsigned char *base = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    unsigned char *sB = base;
    unsigned char *sA = base + round1k(b_bytes(N, KC));
    uint64_t *bars = (uint64_t *)(sA + (size_t)S * KC * A_CHUNK_BYTES);
    uint64_t *full = bars;         // [S]
    uint64_t *mma_bar = bars + S;  // [1]
    uint64_t *b_bar = bars + S + 1;
    uint32_t *tslot = (uint32_t *)(bars + S + 2);
    int *abort_flag = (int *)(tslot + 1);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const long long ntiles = (M + TILE_M - 1) / TILE_M;
    const long long my_tiles = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    constexpr uint32_t NCOLS = tmem_cols(N);
    constexpr uint32_t IDESC = idesc_bf16_f32(N);
    constexpr uint32_t STAGE_TX = KC * A_CHUNK_BYTES;

    if (tid == 0) {
        for (int i = 0; i < S; i++) mbar_init(&full[i], 1);
        mbar_init(mma_bar, 1);
        mbar_init(b_bar, 1);
        *abort_flag = 0;
        fence_mbar_init();
    }
    if (warp == 0) {
        tmem_alloc(tslot, NCOLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t taddr = *tslot;

    long long issued = 0;  // A tiles whose loads thread 0 has issued
    if (tid == 0 && my_tiles > 0) {
        mbar_expect_tx(b_bar, (uint32_t)b_bytes(N, KC));
        for (int kc = 0; kc < KC; kc++) tma_load_2d(sB + (size_t)kc * N * 64, &tb, b_bar, kc * KCHUNK, 0);
        for (; issued < my_tiles && issued < S - 1; issued++) {
            const int st = (int)(issued % S);
            const long long t = blockIdx.x + issued * gridDim.x;
            mbar_expect_tx(&full[st], STAGE_TX);
            for (int kc = 0; kc < KC; kc++)
                tma_load_2d(sA + ((size_t)st * KC + kc) * A_CHUNK_BYTES, &ta, &full[st], kc * KCHUNK,
                            (int)(t * TILE_M));
        }
    }

    long long i = 0;
    for (; i < my_tiles; i++) {
        const long long t = blockIdx.x + i * gridDim.x;
        if (tid == 0) {
            bool ok = true;
            if (i == 0) ok = mbar_wait(b_bar, 0);
            if (ok && issued < my_tiles) {  // refill the stage tile i-1 used (its MMA has completed)
                const int st = (int)(issued % S);
                const long long tt = blockIdx.x + issued * gridDim.x;
                mbar_expect_tx(&full[st], STAGE_TX);
                for (int kc = 0; kc < KC; kc++)
                    tma_load_2d(sA + ((size_t)st * KC + kc) * A_CHUNK_BYTES, &ta, &full[st], kc * KCHUNK,
                                (int)(tt * TILE_M));
                issued++;
            }
            const int st = (int)(i % S);
            if (ok) ok = mbar_wait(&full[st], (uint32_t)((i / S) & 1));
            if (ok) {
                tc_fence_after();
                const uint32_t a0 = smem_u32(sA + (size_t)st * KC * A_CHUNK_BYTES), b0 = smem_u32(sB);
#pragma unroll
                for (int kc = 0; kc < KC; kc++)
#pragma unroll
                    for (int kk = 0; kk < 2; kk++)
                        mma_bf16(taddr, desc_k_sw64(a0 + kc * A_CHUNK_BYTES + kk * 32),
                                 desc_k_sw64(b0 + kc * N * 64 + kk * 32), IDESC, (kc | kk) ? 1u : 0u);
                mma_commit(mma_bar);
            } else {
                *abort_flag = 1;
            }
        }
        __syncthreads();
        if (*abort_flag) break;
        const bool ok = mbar_wait(mma_bar, (uint32_t)(i & 1));
        if (!ok) *abort_flag = 1;  // benign race: every writer stores 1
        __syncthreads();
        if (*abort_flag) break;
        tc_fence_after();
        const long long row = t * TILE_M + warp * 32 + lane;
        const uint32_t trow = taddr + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
        for (int c0 = 0; c0 < N; c0 += 32) {
            float acc[32];
            __syncwarp();
            tmem_ld32(trow + c0, acc);
            if (row < M) e.row(row, acc, c0);
        }
        if (row < M) e.done(row);
        tc_fence_before();
        __syncthreads();
    }

    if (*abort_flag) {
        if (tid == 0) {
            atomicExch(err, 1);
            // let this CTA's own loads in flight land before its shared memory goes away
            for (long long q = i; q < issued; q++) mbar_wait(&full[q % S], (uint32_t)((q / S) & 1));
            if (i == 0 && my_tiles > 0) mbar_wait(b_bar, 0);
        }
        __syncthreads();
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(taddr, NCOLS);
    }
}

}  // namespace umma
}  // namespace cg
