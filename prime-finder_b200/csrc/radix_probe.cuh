// Two forms of one radix-16 pass of the squaring kernel's transform, for
// measurement (pfb_mr_radix16_forms): the first forward pass of a 2^14-point
// transform, both primes, from the same 2^14 limbs of 22 bits.
//
//   butterfly  the engine's own pass (dif_pass_t: four radix-2 stages with
//              Shoup twiddles on the integer pipe)
//   tensor     the same pass as an exact int8 matrix product on the 5th-
//              generation tensor cores (tcgen05.mma kind::i8, accumulators in
//              tensor memory), then recombination on the CUDA cores
//
// The pass maps position j0 + e 2^10 (e < 16) to
//   y = omega_n^(j0 k) sum_m x[j0 + m 2^10] omega_16^(m k),  k = bitrev4(e),
// a DFT of length 16 followed by a twiddle.  The tensor form splits the DFT
// matrix F (entries < 2^30) into 4 byte planes F_b and the limbs (< 2^22)
// into 3 byte planes x_a: A = the 128 rows (prime, k, b) of F_b, B_a = the
// byte plane a of 128 groups j0, K = 16 values of m padded to the
// instruction's 32; D_a = A B_a^T (exact: 16 * 255 * 255 < 2^20).  Then per
// output y = omega_n^(j0 k) sum_(a,b) 2^(8(a+b)) D_a[(prime, k, b), j0] mod p.
// Nothing here is on the Miller-Rabin path: the butterfly pass is what the
// squaring kernel runs; the tensor form exists to measure against it.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "mr_device.cuh"

namespace pfb {
namespace mr {

constexpr int RP_LOGN = 14, RP_N = 1 << RP_LOGN, RP_SUB = RP_N / 16, RP_TILE = 128;
constexpr int RP_TILES = RP_SUB / RP_TILE;        // 8 tiles of 128 groups
constexpr int RP_OPND = 4096;                      // bytes of one operand image (128 rows x 32 bytes)
constexpr int RP_TMEM_COLS = 512;                  // 3 planes x 128 columns, rounded to a power of two
// x, A, 3 B planes, barrier; padded past half the SM's shared memory so that
// one CTA per SM holds all of tensor memory and no second CTA waits in alloc
constexpr int RP_SMEM = RP_N * 4 + 4 * RP_OPND + 256 + 40960;

struct RpTables {
    const uint8_t *fa;                 // A operand image: 128 rows (prime, k, b) x 32 bytes, K-major core matrices
    const uint32_t *wn[2], *wnsh[2];   // omega_n^t (t < n) per prime, and Shoup companions
    unsigned long long mu[2];          // floor(2^64 / p)
};

// The engine's pass: both primes, two halves of the CTA.
__global__ void __launch_bounds__(THREADS, 1) rp_butterfly_kernel(const uint32_t *x, uint32_t *y, Twiddles tw) {
    PFB_DYNAMIC_SMEM(uint32_t, raw);
    uint32_t *A0 = raw, *A1 = raw + RP_N + RP_N / 32;
    const uint32_t *xb = x + (size_t)blockIdx.x * RP_N;
    uint32_t *yb = y + (size_t)blockIdx.x * 2 * RP_N;
    for (int i = threadIdx.x; i < RP_N; i += THREADS) {
        const uint32_t v = xb[i];
        A0[pad(i)] = v;
        A1[pad(i)] = v;
    }
    __syncthreads();
    constexpr int half = THREADS / 2;
    if ((int)threadIdx.x < half) dif_pass_t<0, 4, RP_LOGN, RP_LOGN - 1, half>(A0, tw.w[0], tw.wsh[0], threadIdx.x);
    else dif_pass_t<1, 4, RP_LOGN, RP_LOGN - 1, half>(A1, tw.w[1], tw.wsh[1], threadIdx.x - half);
    __syncthreads();
    for (int i = threadIdx.x; i < RP_N; i += THREADS) {
        yb[i] = red2(A0[pad(i)], P1);
        yb[RP_N + i] = red2(A1[pad(i)], P2);
    }
}

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor, K-major, no swizzle: 8-row x 16-byte core
// matrices, the two K halves 128 bytes apart (leading offset), 8-row groups
// 256 bytes apart (stride offset), descriptor version 1.
__device__ __forceinline__ unsigned long long rp_desc(uint32_t saddr) {
    return (unsigned long long)((saddr >> 4) & 0x3FFFu) | (8ull << 16) | (16ull << 32) | (1ull << 46);
}

// Byte offset of (row, m) in an operand image (m < 32).
__host__ __device__ __forceinline__ int rp_off(int row, int m) {
    return (row >> 3) * 256 + (m >> 4) * 128 + (row & 7) * 16 + (m & 15);
}

__device__ __forceinline__ uint32_t rp_mod(unsigned long long v, uint32_t p, unsigned long long mu) {
    unsigned long long r = v - __umul64hi(v, mu) * p;
    while (r >= p) r -= p;
    return (uint32_t)r;
}

// Instruction descriptor: kind::i8, D s32, A and B unsigned 8-bit K-major, M = 128, N = 128.
constexpr uint32_t RP_IDESC = (2u << 4) | ((128u >> 3) << 17) | ((128u >> 4) << 24);

__global__ void __launch_bounds__(THREADS, 1)
rp_tensor_kernel(const uint32_t *x, uint32_t *y, RpTables t, int *err) {
    extern __shared__ __align__(1024) uint8_t rp_raw[];
    uint32_t *xs = reinterpret_cast<uint32_t *>(rp_raw);
    uint8_t *sa = rp_raw + RP_N * 4;
    uint8_t *sb = sa + RP_OPND;
    unsigned long long *mbar = reinterpret_cast<unsigned long long *>(sb + 3 * RP_OPND);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(mbar + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t *xb = x + (size_t)blockIdx.x * RP_N;
    uint32_t *yb = y + (size_t)blockIdx.x * 2 * RP_N;
    for (int i = tid; i < RP_N; i += THREADS) xs[i] = xb[i];
    for (int i = tid; i < RP_OPND / 16; i += THREADS)
        reinterpret_cast<uint4 *>(sa)[i] = reinterpret_cast<const uint4 *>(t.fa)[i];
    for (int i = tid; i < 3 * RP_OPND / 16; i += THREADS) reinterpret_cast<uint4 *>(sb)[i] = make_uint4(0, 0, 0, 0);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tslot)),
                     "r"(RP_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(mbar)));
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = *tslot;
    const unsigned long long da = rp_desc(smem_addr(sa));
    uint32_t phase = 0;
    bool ok = true;
    const int q = warp & 3, cb = warp >> 2;  // lane quadrant, block of 32 columns
    const int row = 32 * q + lane, pr = row >> 6, k = (row & 63) >> 2, b = row & 3;
    const uint32_t p = pr ? P2 : P1;
    const int kr = ((k & 1) << 3) | ((k & 2) << 1) | ((k & 4) >> 1) | ((k & 8) >> 3);  // bitrev4(k)
    for (int tile = 0; tile < RP_TILES && ok; tile++) {
        // byte planes of the tile's 128 groups
        for (int idx = tid; idx < RP_TILE * 16; idx += THREADS) {
            const int g = idx >> 4, m = idx & 15;
            const uint32_t v = xs[tile * RP_TILE + g + m * RP_SUB];
            const int o = rp_off(g, m);
            sb[o] = (uint8_t)v;
            sb[RP_OPND + o] = (uint8_t)(v >> 8);
            sb[2 * RP_OPND + o] = (uint8_t)(v >> 16);
        }
        asm volatile("fence.proxy.async.shared::cta;");
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;");
        if (tid == 0) {
            for (int a = 0; a < 3; a++) {
                const unsigned long long db = rp_desc(smem_addr(sb + a * RP_OPND));
                const uint32_t d = tmem + (uint32_t)(a * RP_TILE), z = 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d),
                    "l"(da), "l"(db), "r"(RP_IDESC), "r"(0u), "r"(z), "r"(z), "r"(z), "r"(z));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                smem_addr(mbar)));
        }
        // bounded wait for the three products
        uint32_t done = 0;
        for (int it = 0; it < (1 << 22) && !done; it++)
            asm volatile(
                "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                "selp.u32 %0, 1, 0, p;\n\t}\n"
                : "=r"(done)
                : "r"(smem_addr(mbar)), "r"(phase));
        phase ^= 1u;
        if (!__syncthreads_and(done != 0)) {
            if (tid == 0) atomicExch(err, 1);
            ok = false;
            break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;");
        // each thread: row (prime, k, b) of the accumulators, 32 columns (groups)
        for (int h = 0; h < 2; h++) {
            const int col0 = cb * 32 + h * 16;
            uint32_t v[3][16];
            for (int a = 0; a < 3; a++) {
                const uint32_t ta = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(a * RP_TILE + col0);
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                    "[%16];"
                    : "=r"(v[a][0]), "=r"(v[a][1]), "=r"(v[a][2]), "=r"(v[a][3]), "=r"(v[a][4]), "=r"(v[a][5]),
                      "=r"(v[a][6]), "=r"(v[a][7]), "=r"(v[a][8]), "=r"(v[a][9]), "=r"(v[a][10]), "=r"(v[a][11]),
                      "=r"(v[a][12]), "=r"(v[a][13]), "=r"(v[a][14]), "=r"(v[a][15])
                    : "r"(ta));
            }
            asm volatile("tcgen05.wait::ld.sync.aligned;");
#pragma unroll
            for (int c = 0; c < 16; c++) {
                const unsigned long long part = ((unsigned long long)v[0][c] << (8 * b)) +
                                                ((unsigned long long)v[1][c] << (8 * b + 8)) +
                                                ((unsigned long long)v[2][c] << (8 * b + 16));
                uint32_t r = rp_mod(part, p, t.mu[pr]);
                r += __shfl_xor_sync(0xffffffffu, r, 1);  // < 2p
                r += __shfl_xor_sync(0xffffffffu, r, 2);  // < 4p < 2^32
                r = red2(red2(r, 2u * p), p);
                if (b == 0) {
                    const int j0 = tile * RP_TILE + col0 + c;
                    const int e = (j0 * k) & (RP_N - 1);
                    const uint32_t o = red2(shoup(r, __ldg(t.wn[pr] + e), __ldg(t.wnsh[pr] + e), p), p);
                    yb[pr * RP_N + j0 + kr * RP_SUB] = o;
                }
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;");
    }
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(RP_TMEM_COLS));
}

}  // namespace mr
}  // namespace pfb
