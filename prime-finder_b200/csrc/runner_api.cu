// The reference's C++ Miller-Rabin surface (BatchModCtx, gpu_miller_rabin[_s1],
// miller_rabin.h's miller_rabin_test) implemented on the pfb_mr engine.
#include <stdint.h>
#include <stdio.h>

#include <chrono>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "batch_mod_ctx.cuh"
#include "common.cuh"
#include "bigint_host.h"
#include "phase2_host.h"
#include "miller_rabin.h"
#include "miller_rabin_runner.cuh"
#include "pfb_mr.h"

BatchModCtx::BatchModCtx(const std::vector<uint64_t> &N_all, int n_limbs_, int n_batch_, int device_id_)
    : n_limbs(n_limbs_), n_batch(n_batch_), n_sum(2 * n_limbs_ + 16), device_id(device_id_) {
    if (n_limbs <= 0 || n_batch <= 0 || N_all.size() < (size_t)n_limbs * (size_t)n_batch)
        throw std::runtime_error("BatchModCtx: N_all holds fewer than n_batch * n_limbs limbs");
    N16.resize((size_t)n_limbs * n_batch);
    for (size_t i = 0; i < N16.size(); i++) {
        if (N_all[i] > 0xFFFFu) throw std::runtime_error("BatchModCtx: limbs must be 16-bit values");
        N16[i] = (uint16_t)N_all[i];
    }
    if (pfb_mr_create(&engine, device_id) != PFB_OK)
        throw std::runtime_error(std::string("BatchModCtx: ") + pfb_last_error());
    if (pfb_mr_ctx_create(engine, N_all.data(), n_limbs, n_batch, &ctx) != PFB_OK ||
        pfb_mr_ctx_buffers(ctx, &d_N, &d_one_res, &d_Nm1_res) != PFB_OK) {
        const std::string msg = std::string("BatchModCtx: ") + pfb_last_error();
        pfb_mr_ctx_destroy(ctx);
        pfb_mr_destroy(engine);
        throw std::runtime_error(msg);
    }
}

BatchModCtx::~BatchModCtx() {
    pfb_mr_ctx_destroy(ctx);
    pfb_mr_destroy(engine);
}

namespace {

void ctx_check(int rc, const char *what) {
    if (rc != PFB_OK) throw std::runtime_error(std::string(what) + ": " + pfb_last_error());
}

}  // namespace

void BatchModCtx::to_residue_batch(const std::vector<uint64_t> &x_all, std::vector<uint64_t> &out_all) const {
    if (x_all.size() < (size_t)n_batch * n_limbs) throw std::runtime_error("to_residue_batch: x_all too short");
    out_all.assign((size_t)n_batch * n_limbs, 0);
    ctx_check(pfb_mr_ctx_to_residue(ctx, x_all.data(), out_all.data()), "to_residue_batch");
}

void BatchModCtx::from_residue_batch(const Data64 *d_x, std::vector<uint64_t> &out_all) const {
    out_all.assign((size_t)n_batch * n_limbs, 0);
    ctx_check(pfb_mr_ctx_from_residue(ctx, d_x, out_all.data()), "from_residue_batch");
}

void BatchModCtx::check_passed(const Data64 *d_r_mont, uint8_t *d_passed, cudaStream_t s) const {
    ctx_check(pfb_mr_ctx_check_passed(ctx, d_r_mont, d_passed, s), "check_passed");
}

void BatchModCtx::modmul_batch(const Data64 *d_A, const Data64 *d_B, Data64 *d_out, cudaStream_t s) {
    ctx_check(pfb_mr_ctx_modmul(ctx, d_A, d_B, d_out, s), "modmul_batch");
}

void BatchModCtx::modsq_batch(const Data64 *d_A, Data64 *d_out, cudaStream_t s) {
    ctx_check(pfb_mr_ctx_modsq(ctx, d_A, d_out, s), "modsq_batch");
}

void BatchModCtx::mul_no_redc_batch(const Data64 *d_A, const Data64 *d_B, Data64 *d_out, cudaStream_t s) {
    ctx_check(pfb_mr_ctx_mul_raw(ctx, d_A, d_B, d_out, s), "mul_no_redc_batch");
    ctx_check(cudaStreamSynchronize(s) == cudaSuccess ? PFB_OK : PFB_E_CUDA, "mul_no_redc_batch");
}

void BatchModCtx::sq_no_redc_batch(const Data64 *d_A, Data64 *d_out, cudaStream_t s) {
    ctx_check(pfb_mr_ctx_sq_raw(ctx, d_A, d_out, s), "sq_no_redc_batch");
    ctx_check(cudaStreamSynchronize(s) == cudaSuccess ? PFB_OK : PFB_E_CUDA, "sq_no_redc_batch");
}

namespace {

std::vector<bool> run_witnesses(BatchModCtx &mont, int n_total, const std::vector<uint32_t> &witnesses,
                                const char *label, bool show_report) {
    if (n_total < 0 || n_total > mont.n_batch) throw std::runtime_error("gpu_miller_rabin: n_total > n_batch");
    std::vector<bool> alive(n_total, true);
    for (uint32_t w : witnesses) {
        std::vector<int> idx;
        for (int t = 0; t < n_total; t++)
            if (alive[t]) idx.push_back(t);
        if (idx.empty()) break;
        if (show_report) printf("  [%s] witness %-3u alive: %zu\n", label ? label : "", w, idx.size());
        std::vector<pfb_mr_number_t> nums(idx.size());
        for (size_t i = 0; i < idx.size(); i++)
            nums[i] = pfb_mr_number_t{mont.N16.data() + (size_t)idx[i] * mont.n_limbs, mont.n_limbs};
        std::vector<int8_t> ver(idx.size());
        if (pfb_mr_test(mont.engine, nums.data(), (int)nums.size(), w, ver.data(), nullptr, 0) != PFB_OK)
            throw std::runtime_error(std::string("gpu_miller_rabin: ") + pfb_last_error());
        for (size_t i = 0; i < idx.size(); i++)
            if (ver[i] != 1) alive[idx[i]] = false;
    }
    return alive;
}

}  // namespace

std::vector<bool> gpu_miller_rabin_s1(BatchModCtx &mont, const std::vector<uint64_t> &, const std::vector<uint64_t> &,
                                      int n_total, const std::vector<uint32_t> &witnesses, const char *label,
                                      bool show_report, bool) {
    return run_witnesses(mont, n_total, witnesses, label, show_report);
}

std::vector<bool> gpu_miller_rabin(BatchModCtx &mont, const std::vector<uint64_t> &, const std::vector<uint64_t> &,
                                   int, int n_total, const std::vector<uint32_t> &witnesses, const char *label,
                                   bool show_report, bool) {
    return run_witnesses(mont, n_total, witnesses, label, show_report);
}

// ---------------------------------------------------------------------------
// miller_rabin_test: one engine per device, created on first use.

namespace {

std::mutex g_mu;
std::vector<pfb_mr_t *> g_eng;

double secs(std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
    return std::chrono::duration<double>(b - a).count();
}

}  // namespace

extern "C" int pfb_mr_bpsw(pfb_mr_t *e, const pfb_mr_number_t *nums, int n, int8_t *verdict) {
    if (!e || !nums || n <= 0 || !verdict) {
        pfb::set_error("pfb_mr_bpsw: bad argument");
        return PFB_E_ARG;
    }
    std::vector<pfb::big::Words> w(n);
    for (int i = 0; i < n; i++) {
        if (!nums[i].limbs || nums[i].n_limbs <= 0) {
            pfb::set_error("pfb_mr_bpsw: number %d has no limbs", i);
            return PFB_E_ARG;
        }
        w[i] = pfb::big::from_u16(nums[i].limbs, (size_t)nums[i].n_limbs);
    }
    const std::vector<int> v = pfb::phase2::prp_batch(e, w);
    if (v.empty()) return PFB_E_CUDA;
    for (int i = 0; i < n; i++) verdict[i] = (int8_t)v[i];
    return PFB_OK;
}

extern "C" int miller_rabin_test(long long a, long long b, long long c, int k, int j, mr_timing_t *timing) {
    if (timing) *timing = mr_timing_t{0.0, 0.0, 0.0, 0.0};
    if (k < 1 || j < 1 || k > 9999 || j > 9999) return -1;
    pfb_mr_t *e = nullptr;
    {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess) return -1;
        std::lock_guard<std::mutex> lk(g_mu);
        if ((int)g_eng.size() <= dev) g_eng.resize(dev + 1, nullptr);
        if (!g_eng[dev] && pfb_mr_create(&g_eng[dev], dev) != PFB_OK) return -1;
        e = g_eng[dev];
    }
    using clk = std::chrono::steady_clock;
    const auto t0 = clk::now();
    const pfb::big::Words N = pfb::phase2::build_n(a, b, c, k, j);
    const auto t1 = clk::now();
    if (N.empty()) return -1;
    const std::vector<int> vN = pfb::phase2::prp_batch(e, {N});
    const int rN = vN.empty() ? -1 : vN[0];
    const auto t2 = clk::now();
    if (timing) {
        timing->build_n = secs(t0, t1);
        timing->mr_n = secs(t1, t2);
    }
    if (rN <= 0) return rN;
    const pfb::big::Words R = pfb::phase2::build_rev(a, b, c, k, j);
    const auto t3 = clk::now();
    if (R.empty()) return -1;
    const std::vector<int> vR = pfb::phase2::prp_batch(e, {R});
    const int rR = vR.empty() ? -1 : vR[0];
    const auto t4 = clk::now();
    if (timing) {
        timing->build_revn = secs(t2, t3);
        timing->mr_revn = secs(t3, t4);
    }
    if (rR < 0) return -1;
    return rR ? 2 : 1;
}
