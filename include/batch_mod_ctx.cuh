// batch_mod_ctx.cuh — C++ surface of the reference's BatchModCtx.
//
// Same public constructors, members callers read, and methods as
// miller_rabin_gpu/batch_mod_ctx.cuh:52-179 (non-copyable, throws
// std::runtime_error on failure, device buffers of 16-bit limbs stored one
// per uint64 -- the reference's Data64 layout -- n_batch moduli back to
// back), so the reference's callers (bench_mr_gpu.cu:48-66,
// helpers/bench_ops.cu, correctness_tests.cuh) compile against it.  Each
// method is one call of the B200 engine's modular context (pfb_mr.h,
// pfb_mr_ctx_*): one CTA per modulus runs a whole Montgomery product --
// forward transforms, pointwise product, inverse transforms, reduction and
// carries -- where the reference chains about 39 launches per product.
//
// Working form: x R mod N, fully reduced, R = 2^(22 H) for the modulus'
// transform length H (the reference's own working form is a Montgomery or
// Barrett residue with its own R; callers only pass it between these
// methods).  The reference's reduction-specific internals (the Multiplier
// object `ntt`, Barrett's mu, the perf-timer tree) have no counterpart.
//
// Plain C++ with the CUDA runtime API header for cudaStream_t.  The mpz_t
// constructor is available when <gmp.h> is on the include path, as in the
// reference, which requires it.
#pragma once
#include <cuda_runtime_api.h>

#include <algorithm>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "pfb_mr.h"

#if __has_include(<gmp.h>)
#include <gmp.h>
#define PFB_BATCH_MOD_CTX_GMP 1
#endif

typedef uint64_t Data64;  // one 16-bit limb per word (the reference's device layout)

struct BatchModCtx {
    int n_limbs = 0;  // 16-bit limbs per modulus (ntt_merge.cuh:14-24)
    int n_batch = 0;  // number of moduli
    int n_sum = 0;    // limbs of a raw product: 2 n_limbs + 16 (batch_mod_ctx.cu:85)
    int device_id = 0;
    bool perf_enabled = false;  // accepted for source compatibility; timing is ncu's job here

    // Device copies owned by the context (read-only for callers): N, and the
    // working forms of 1 and N - 1, [n_batch * n_limbs] each.
    const Data64 *d_N = nullptr;
    const Data64 *d_one_res = nullptr;
    const Data64 *d_Nm1_res = nullptr;

    pfb_mr_t *engine = nullptr;
    pfb_mr_ctx_t *ctx = nullptr;
    std::vector<uint16_t> N16;  // n_batch * n_limbs little-endian 16-bit limbs

    // N_all: flat [n_batch * n_limbs], 16-bit limbs stored in uint64.
    explicit BatchModCtx(const std::vector<uint64_t> &N_all, int n_limbs_, int n_batch_, int device_id_ = 0);
#ifdef PFB_BATCH_MOD_CTX_GMP
    // The numbers as mpz_t; n_limbs = limbs_for_digits(max decimal digits + 4)
    // as in batch_mod_ctx.cu:52-80.
    explicit BatchModCtx(const std::vector<mpz_t *> &numbers, int device_id_ = 0)
        : BatchModCtx(gmp_limbs(numbers), gmp_n_limbs(numbers), (int)numbers.size(), device_id_) {}
#endif
    ~BatchModCtx();
    BatchModCtx(const BatchModCtx &) = delete;
    BatchModCtx &operator=(const BatchModCtx &) = delete;

    // x_all (host, n_batch * n_limbs) -> working form (host)
    void to_residue_batch(const std::vector<uint64_t> &x_all, std::vector<uint64_t> &out_all) const;
    // d_x (device, working form) -> plain values (host); synchronises
    void from_residue_batch(const Data64 *d_x, std::vector<uint64_t> &out_all) const;
    // d_passed[t] = 1 when d_r_mont[t] is the working form of 1 or N - 1
    void check_passed(const Data64 *d_r_mont, uint8_t *d_passed, cudaStream_t s = 0) const;
    // d_out = a b / a^2 in the working form, every modulus
    void modmul_batch(const Data64 *d_A, const Data64 *d_B, Data64 *d_out, cudaStream_t s = 0);
    void modsq_batch(const Data64 *d_A, Data64 *d_out, cudaStream_t s = 0);
    // d_out = the full product (n_sum limbs per modulus), no reduction; synchronises
    // like the reference (batch_mod_ctx.cu:320-335)
    void mul_no_redc_batch(const Data64 *d_A, const Data64 *d_B, Data64 *d_out, cudaStream_t s = 0);
    void sq_no_redc_batch(const Data64 *d_A, Data64 *d_out, cudaStream_t s = 0);

#ifdef PFB_BATCH_MOD_CTX_GMP
  private:
    // limbs_for_digits (ntt_merge.cuh:21-24) of the widest number + 4 digits
    static int gmp_n_limbs(const std::vector<mpz_t *> &numbers) {
        int d = 0;
        for (auto *p : numbers) d = std::max(d, (int)mpz_sizeinbase(*p, 10));
        return (int)(((d + 4) * 3.32193 + 15) / 16) + 4;
    }
    static std::vector<uint64_t> gmp_limbs(const std::vector<mpz_t *> &numbers) {
        const int nl = gmp_n_limbs(numbers);
        std::vector<uint64_t> all((size_t)nl * numbers.size(), 0);
        std::vector<uint16_t> w((size_t)nl + 8);
        for (size_t i = 0; i < numbers.size(); i++) {
            size_t cnt = 0;
            std::fill(w.begin(), w.end(), 0);
            if (mpz_sizeinbase(*numbers[i], 2) > 16 * (size_t)nl)
                throw std::runtime_error("BatchModCtx: number wider than n_limbs");
            mpz_export(w.data(), &cnt, -1, 2, 0, 0, *numbers[i]);
            for (int k = 0; k < nl; k++) all[i * nl + k] = w[k];
        }
        return all;
    }
#endif
};
