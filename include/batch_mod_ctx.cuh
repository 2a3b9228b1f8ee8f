// batch_mod_ctx.cuh — C++ surface of the reference's BatchModCtx.
//
// Same public constructor and sizes as miller_rabin_gpu/batch_mod_ctx.cuh:
// 101-228 (`BatchModCtx(const std::vector<uint64_t>& N_all, int n_limbs,
// int n_batch, int device_id = 0)`, non-copyable, throws std::runtime_error
// on failure), so callers such as bench_mr_gpu.cu:48-66 compile unchanged.
// Inside, the moduli are handed to the B200 engine of pfb_mr.h; the
// reference's per-operation methods (modsq_batch, modmul_batch, residue
// conversions) have no counterpart here: the engine runs whole
// exponentiations on chip.  Plain C++ (no CUDA syntax).
#pragma once
#include <cstdint>
#include <vector>

#include "pfb_mr.h"

struct BatchModCtx {
    int n_limbs = 0;      // 16-bit limbs per modulus (ntt_merge.cuh:14-24)
    int n_batch = 0;      // number of moduli
    int device_id = 0;
    bool perf_enabled = false;
    pfb_mr_t *engine = nullptr;
    std::vector<uint16_t> N16;  // n_batch * n_limbs little-endian 16-bit limbs

    // N_all: flat [n_batch * n_limbs], 16-bit limbs stored in uint64 (the
    // reference's layout).
    explicit BatchModCtx(const std::vector<uint64_t> &N_all, int n_limbs_, int n_batch_, int device_id_ = 0);
    ~BatchModCtx();
    BatchModCtx(const BatchModCtx &) = delete;
    BatchModCtx &operator=(const BatchModCtx &) = delete;
};
