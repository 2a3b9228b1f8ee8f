// Phase 1 -> Phase 2 on one GPU (pfb_pipeline.h): the sieve's device masks
// are compacted on the device, the survivors' N are built on the host from
// powers of ten cached per triple, and every base-2 strong test runs through
// one continuous-batching server; the rare base-2 probable primes get the
// remaining rounds and their rev(N) in batched engine calls.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <chrono>
#include <map>
#include <vector>

#include "common.cuh"
#include "phase2_host.h"
#include "pfb_mr.h"
#include "pfb_pipeline.h"
#include "pfb_sieve.h"

namespace {

using pfb::big::Words;

struct Survivor {
    int t;     // triple index
    int k, j;
};

struct DevBuf {
    void *p = nullptr;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
};

struct Stream {
    cudaStream_t s = nullptr;
    ~Stream() {
        if (s) cudaStreamDestroy(s);
    }
};

// Powers of ten of one triple, computed on first use.
struct TenPowers {
    std::map<long long, Words> m;
    const Words &get(long long e) {
        auto it = m.find(e);
        if (it == m.end()) it = m.emplace(e, pfb::big::pow10((uint64_t)e)).first;
        return it->second;
    }
};

double secs_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// Phase 1: survivors of every triple, in triple order, k-major.
int sieve_all(pfb_sieve_t *sv, const long long *abc, int n_abc, int K, int per_call, const uint8_t *pre_mask,
              std::vector<Survivor> &surv) {
    const size_t blk = pfb_sieve_mask_bytes(K);
    const size_t cells = (size_t)K * (size_t)K;
    DevBuf d_mask, d_list;
    Stream st;
    PFB_CUDA(cudaStreamCreateWithFlags(&st.s, cudaStreamNonBlocking));
    PFB_CUDA(cudaMalloc(&d_mask.p, blk * (size_t)per_call));
    PFB_CUDA(cudaMalloc(&d_list.p, cells * sizeof(uint32_t)));
    std::vector<uint32_t> list;
    for (int t0 = 0; t0 < n_abc; t0 += per_call) {
        const int n = std::min(per_call, n_abc - t0);
        unsigned flags = 0;
        if (pre_mask) {  // copy, sieve, compaction and read-back all on st, in order
            PFB_CUDA(cudaMemcpyAsync(d_mask.p, pre_mask + (size_t)t0 * blk, blk * (size_t)n, cudaMemcpyHostToDevice,
                                     st.s));
            flags = PFB_SIEVE_OR;
        }
        int rc = pfb_sieve_run(sv, abc + 3 * (size_t)t0, n, K, (uint8_t *)d_mask.p, flags, st.s);
        if (rc) return rc;
        for (int i = 0; i < n; i++) {
            uint32_t count = 0;
            rc = pfb_sieve_survivors(sv, (const uint8_t *)d_mask.p + (size_t)i * blk, K, (uint32_t *)d_list.p,
                                     (uint32_t)cells, &count, st.s);
            if (rc) return rc;
            list.resize(count);
            if (count) {
                PFB_CUDA(cudaMemcpyAsync(list.data(), d_list.p, count * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                         st.s));
                PFB_CUDA(cudaStreamSynchronize(st.s));
            }
            for (uint32_t q : list) surv.push_back(Survivor{t0 + i, (int)(q >> 16), (int)(q & 0xFFFFu)});
        }
    }
    PFB_CUDA(cudaStreamSynchronize(st.s));
    return PFB_OK;
}

}  // namespace

extern "C" int pfb_pipeline_run(pfb_sieve_t *sv, pfb_mr_t *mr, const long long *abc, int n_abc,
                                const pfb_pipeline_config_t *cfg, const uint8_t *pre_mask,
                                pfb_phase2_record_t *out, long long cap, long long *n_out,
                                pfb_pipeline_stats_t *stats) {
    using namespace pfb::phase2;
    using clk = std::chrono::steady_clock;
    if (!sv || !mr || !abc || n_abc <= 0 || !cfg || !n_out || (cap > 0 && !out) || cap < 0) {
        pfb::set_error("pfb_pipeline_run: bad argument");
        return PFB_E_ARG;
    }
    const int K = cfg->K;
    if (K < 1 || K > PFB_SIEVE_MAX_K) {
        pfb::set_error("pfb_pipeline_run: K = %d outside [1, %d]", K, PFB_SIEVE_MAX_K);
        return PFB_E_ARG;
    }
    for (int t = 0; t < 3 * n_abc; t++)
        if (abc[t] < 0) {
            pfb::set_error("pfb_pipeline_run: negative exponent in triple %d", t / 3);
            return PFB_E_ARG;
        }
    *n_out = 0;
    pfb_pipeline_stats_t st{};
    st.triples = n_abc;
    const auto t_start = clk::now();
    const int dev = pfb_mr_device(mr);
    PFB_CUDA(cudaSetDevice(dev));

    // ---- Phase 1 --------------------------------------------------------
    std::vector<Survivor> surv;
    int rc = sieve_all(sv, abc, n_abc, K, cfg->triples_per_sieve > 0 ? cfg->triples_per_sieve : 8, pre_mask, surv);
    if (rc) return rc;
    st.sieve_s = secs_since(t_start);
    const long long total = (long long)surv.size();
    st.survivors = total;
    *n_out = total;
    if (total > cap) {
        pfb::set_error("pfb_pipeline_run: %lld survivors, room for %lld records", total, cap);
        if (stats) *stats = st;
        return PFB_E_CAPACITY;
    }
    for (long long i = 0; i < total; i++) {
        const Survivor &s = surv[i];
        out[i] = pfb_phase2_record_t{abc[3 * s.t], abc[3 * s.t + 1], abc[3 * s.t + 2], s.k, s.j, -1};
    }

    // ---- Phase 2a: base-2 strong test of every N through the server -------
    const auto t_p2 = clk::now();
    int sms = 0;
    PFB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    pfb_mr_server_config_t scfg{};
    scfg.max_resident = cfg->max_resident > 0 ? cfg->max_resident : 2 * sms;
    scfg.hbm_budget_bytes = cfg->hbm_budget_bytes;
    scfg.chunk_steps = 0;
    scfg.base = 2;
    scfg.prep_threads = cfg->prep_threads;
    const long long window = cfg->window > 0 ? cfg->window : 4LL * scfg.max_resident;
    std::vector<int> v2(total, -1);  // base-2 verdict per survivor (-1: none)
    if (total > 0) {
        pfb_mr_server_t *srv = nullptr;
        rc = pfb_mr_server_create(mr, &scfg, &srv);
        if (rc) return rc;
        TenPowers tp;
        int tp_triple = -1;
        long long next = 0, inflight = 0;
        std::vector<uint16_t> l16;
        std::vector<pfb_mr_result_t> res(256);
        while (next < total || inflight > 0) {
            while (next < total && inflight < window) {
                const Survivor &s = surv[next];
                if (s.t != tp_triple) {
                    tp = TenPowers();
                    tp_triple = s.t;
                }
                const long long a = abc[3 * s.t], b = abc[3 * s.t + 1], c = abc[3 * s.t + 2];
                const Words N = a >= 1 ? combine(tp.get(a), tp.get(b), (uint64_t)s.k, tp.get(c), (uint64_t)s.j)
                                       : Words();
                if (N.empty()) {
                    st.invalid++;
                    next++;
                    continue;
                }
                l16.assign((pfb::big::bit_length(N) + 15) / 16, 0);
                pfb::big::to_u16(N, l16.data(), l16.size());
                rc = pfb_mr_server_submit(srv, l16.data(), (int)l16.size(), (uint64_t)next, nullptr, 0);
                if (rc) {
                    pfb_mr_server_destroy(srv);
                    return rc;
                }
                next++;
                inflight++;
            }
            if (inflight == 0) break;
            const int n = pfb_mr_server_poll(srv, res.data(), (int)res.size(), 200);
            if (n < 0) {
                pfb_mr_server_destroy(srv);
                return n;
            }
            for (int i = 0; i < n; i++) {
                v2[res[i].tag] = res[i].verdict;
                inflight--;
            }
        }
        pfb_mr_server_destroy(srv);
    }

    // ---- Phase 2b: remaining rounds on base-2 probable primes (and on the
    // numbers the server did not take: even or too long), then rev(N) ------
    std::vector<long long> idx;
    std::vector<Words> nums;
    std::vector<int> passed;
    for (long long i = 0; i < total; i++) {
        if (v2[i] == 0) out[i].result = 0;
        if (v2[i] == 0) continue;
        const Survivor &s = surv[i];
        Words N = build_n(abc[3 * s.t], abc[3 * s.t + 1], abc[3 * s.t + 2], s.k, s.j);
        if (N.empty()) continue;  // counted as invalid above; result stays -1
        idx.push_back(i);
        nums.push_back(std::move(N));
        passed.push_back(v2[i] == 1);
    }
    if (!idx.empty()) {
        const std::vector<int> vN = prp_batch(mr, nums, &passed);
        if (vN.empty()) return PFB_E_CUDA;
        std::vector<long long> ridx;
        std::vector<Words> rnums;
        for (size_t t = 0; t < idx.size(); t++) {
            if (vN[t] <= 0) {
                out[idx[t]].result = vN[t];
                if (vN[t] < 0) st.invalid++;
                continue;
            }
            st.n_prp++;
            const pfb_phase2_record_t &r = out[idx[t]];
            Words R = build_rev(r.a, r.b, r.c, r.k, r.j);
            if (R.empty()) {
                st.invalid++;
                continue;  // result stays -1
            }
            ridx.push_back(idx[t]);
            rnums.push_back(std::move(R));
        }
        if (!ridx.empty()) {
            const std::vector<int> vR = prp_batch(mr, rnums);
            if (vR.empty()) return PFB_E_CUDA;
            for (size_t t = 0; t < ridx.size(); t++) {
                if (vR[t] < 0) {
                    out[ridx[t]].result = -1;
                    st.invalid++;
                    continue;
                }
                out[ridx[t]].result = vR[t] ? 2 : 1;
                st.rev_tested++;
                if (vR[t]) st.both_prp++;
            }
        }
    }
    st.phase2_s = secs_since(t_p2);
    st.total_s = secs_since(t_start);
    if (stats) *stats = st;
    return PFB_OK;
}
