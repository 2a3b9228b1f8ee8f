// miller_rabin_runner.cuh — C++ Miller-Rabin entry points of the reference's
// GPU library (miller_rabin_gpu/miller_rabin_runner.cuh:15-49), same
// declarations, run by the B200 engine (pfb_mr.h).
//
// For each witness in order, every candidate still alive gets one strong
// probable-prime round; the result is alive[t] = passed every round run.  The
// exponent and N-1 arguments keep the reference's signature; the engine
// derives d and s from N itself (N - 1 = 2^s d), so gpu_miller_rabin and
// gpu_miller_rabin_s1 are the same computation.  Throws std::runtime_error on
// failure (miller_rabin_runner.cu:11-14).
#pragma once
#include <cstdint>
#include <vector>

#include "batch_mod_ctx.cuh"

inline const std::vector<uint32_t> DEFAULT_WITNESSES = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53};

std::vector<bool> gpu_miller_rabin_s1(BatchModCtx &mont, const std::vector<uint64_t> &exp_all,
                                      const std::vector<uint64_t> &Nm1_all, int n_total,
                                      const std::vector<uint32_t> &witnesses, const char *label,
                                      bool show_report = false, bool show_progress = false);

std::vector<bool> gpu_miller_rabin(BatchModCtx &mont, const std::vector<uint64_t> &exp_all,
                                   const std::vector<uint64_t> &Nm1_all, int s, int n_total,
                                   const std::vector<uint32_t> &witnesses, const char *label,
                                   bool show_report = false, bool show_progress = false);
