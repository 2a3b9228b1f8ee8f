// Batched Miller-Rabin engine: kernels and host driver.
//
// One CTA per candidate runs its whole chain of Montgomery squarings on chip
// (mr_device.cuh).  The host side does the per-modulus set-up the reference
// does with GMP (barrett.cu:58-107, montgomery.cu:30-45,
// miller_rabin_runner.cu:315-325): N' = -N^-1 mod R, R mod N, N - 1 = 2^s d.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <thread>
#include <vector>

#include "bigint_host.h"
#include "common.cuh"
#include "lucas_host.h"
#include "mr_device.cuh"
#include "mr_tables_host.h"
#include "pfb_mr.h"

#include "mr_ctx_kernels.cuh"
#include "mr_kernels.cuh"
#include "radix_probe.cuh"
#include "mr_prep_host.h"

using namespace pfb::mr;

struct pfb_mr {
    int device = 0;
    int num_sms = 0;
    cudaStream_t stream = nullptr;
    uint32_t *d_tw = nullptr;
    uint32_t *d_wide = nullptr;
    Twiddles tw{};
    // persistent-kernel parameters per transform length (pfb_mr_autotune):
    // steps of one candidate per quantum, steps per launch
    int quantum[LOG_LMAX + 1];
    int chunk[LOG_LMAX + 1];
};

static int build_tables(pfb_mr *e) {
    const int half = 1 << (LOG_LMAX - 1);
    const std::vector<uint32_t> h = twiddle_table();
    PFB_CUDA(cudaMalloc(&e->d_tw, h.size() * sizeof(uint32_t)));
    PFB_CUDA(cudaMemcpy(e->d_tw, h.data(), h.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
    for (int pr = 0; pr < 2; pr++) {
        uint32_t *base = e->d_tw + (size_t)(4 * pr) * half;
        e->tw.w[pr] = base;
        e->tw.wsh[pr] = base + half;
        e->tw.wi[pr] = base + 2 * half;
        e->tw.wish[pr] = base + 3 * half;
    }
    const CrtConsts cc = crt_consts();
    PFB_CUDA(cudaMemcpyToSymbol(c_crt, &cc, sizeof(cc)));
    WideTabs wt{};
    const std::vector<uint32_t> wide = wide_tables(h, wt);
    PFB_CUDA(cudaMalloc(&e->d_wide, wide.size() * sizeof(uint32_t)));
    PFB_CUDA(cudaMemcpy(e->d_wide, wide.data(), wide.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
    wt.base = (const uint4 *)e->d_wide;
    PFB_CUDA(cudaMemcpyToSymbol(c_wide, &wt, sizeof(wt)));
    return PFB_OK;
}

extern "C" int pfb_mr_device(const pfb_mr_t *e) { return e ? e->device : -1; }

extern "C" int pfb_mr_create(pfb_mr_t **out, int device) {
    if (!out) {
        pfb::set_error("pfb_mr_create: null out");
        return PFB_E_ARG;
    }
    *out = nullptr;
    pfb_mr *e = new pfb_mr();
    e->device = device;
    for (int lg = 0; lg <= LOG_LMAX; lg++) {
        e->quantum[lg] = 64;
        e->chunk[lg] = 2048;
    }
    int rc = PFB_OK;
    cudaError_t ce = cudaSetDevice(device);
    if (ce != cudaSuccess) rc = pfb::cuda_fail(ce, "cudaSetDevice", __FILE__, __LINE__);
    if (!rc) {
        ce = cudaDeviceGetAttribute(&e->num_sms, cudaDevAttrMultiProcessorCount, device);
        if (ce != cudaSuccess) rc = pfb::cuda_fail(ce, "attr", __FILE__, __LINE__);
    }
    if (!rc) {
        ce = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
        if (ce != cudaSuccess) rc = pfb::cuda_fail(ce, "stream", __FILE__, __LINE__);
    }
    if (!rc) rc = build_tables(e);
    if (!rc) {
        const int mx = (int)std::max(smem_bytes(LOG_LCTA), smem_bytes(LOG_LSEQ));
        ce = cudaFuncSetAttribute(persist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
        if (ce == cudaSuccess) ce = cudaFuncSetAttribute(prep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
        if (ce == cudaSuccess) ce = cudaFuncSetAttribute(ctx_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
        if (ce != cudaSuccess) rc = pfb::cuda_fail(ce, "smem attribute", __FILE__, __LINE__);
    }
    if (rc) {
        if (e->stream) cudaStreamDestroy(e->stream);
        cudaFree(e->d_tw);
        delete e;
        return rc;
    }
    *out = e;
    return PFB_OK;
}

extern "C" void pfb_mr_destroy(pfb_mr_t *e) {
    if (!e) return;
    cudaSetDevice(e->device);
    if (e->stream) {
        cudaStreamSynchronize(e->stream);
        cudaStreamDestroy(e->stream);
    }
    cudaFree(e->d_tw);
    cudaFree(e->d_wide);
    delete e;
}

namespace {

// Per-candidate device layout inside the arena (32-bit words).
struct Layout {
    size_t x, res, nn, nh, npl, nl, exp, yb, lv0, lv1, lqk, lt, lone, gy, raw, total;
};

Layout layout_for(int logl, size_t exp_words, bool lucas = false, bool raw = false) {
    const size_t L = (size_t)1 << logl, H = L / 2;
    Layout l{};
    size_t o = 0;
    auto take = [&](size_t words) {
        const size_t at = o;
        o += (words + 63) & ~(size_t)63;  // 256-byte alignment
        return at;
    };
    l.x = take(H);
    l.res = take(H);
    l.nn = take(2 * H);
    l.nh = take(2 * H);
    l.npl = take(H);
    l.nl = take(H);
    l.exp = take(exp_words);
    if (logl > LOG_LCTA) l.yb = take(H + H / 32);  // padded like the shared-memory residue
    if (lucas) {
        l.lv0 = take(H);
        l.lv1 = take(H);
        l.lqk = take(H);
        l.lt = take(H);
        l.lone = take(H);
        l.gy = take(2 * L);
    }
    if (raw) l.raw = take(2 * L);  // L 64-bit coefficients
    l.total = o;
    return l;
}

Layout layout_for(const HostPrep &hp, bool lucas) { return layout_for(hp.logl, hp.exp.size(), lucas); }

// Slot layout of the server: the exponent region sized for the longest
// modulus of the length class, so that slots of one class are interchangeable.
Layout slot_layout(int logl) {
    const size_t H = (size_t)1 << (logl - 1);
    return layout_for(logl, (LIMB_BITS * H + 31) / 32 + 1);
}

void prep_all(const pfb_mr_number_t *nums, int n, uint32_t base, int mode, const pfb_mr_number_t *exps,
              std::vector<HostPrep> &hp) {
    hp.resize(n);
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const int nt = (int)std::min<unsigned>(hw, (unsigned)std::max(1, n));
    if (nt <= 1 || n < 4) {
        for (int i = 0; i < n; i++) host_prep(nums[i], base, mode, exps ? exps + i : nullptr, hp[i]);
        return;
    }
    std::vector<std::thread> th;
    for (int t = 0; t < nt; t++)
        th.emplace_back([&, t]() {
            for (int i = t; i < n; i += nt) host_prep(nums[i], base, mode, exps ? exps + i : nullptr, hp[i]);
        });
    for (auto &x : th) x.join();
}

}  // namespace

// A set of candidates resident in device memory, advanced step by step.
struct pfb_mr_batch {
    pfb_mr *e = nullptr;
    int n = 0, mode = 1, maxlog = LOG_LMIN, n_ok = 0;
    long long max_steps = 0, steps_done = 0;
    uint8_t *d_arena = nullptr;
    JobDev *d_jobs = nullptr;
    int *d_locks = nullptr;           // [n] per-candidate locks of the persistent kernel
    unsigned int *d_counter = nullptr;  // quanta handed out in the current launch
    LucasDev *d_lucas = nullptr;        // [n] (strong Lucas batches only)
    std::vector<HostPrep> hp;
    std::vector<JobDev> jobs;
    std::vector<LucasDev> lucas;
    struct Graph {
        long long chunk;
        int quantum;
        cudaGraphExec_t exec;
    };
    std::vector<Graph> graphs;  // one launch of the persistent kernel per (chunk, quantum)
};

namespace {

void batch_free(pfb_mr_batch *b) {
    for (auto &g : b->graphs) cudaGraphExecDestroy(g.exec);
    cudaFree(b->d_arena);
    delete b;
}

// One step chunk of a batch -- the quanta counter reset and the persistent
// kernel -- as a CUDA graph, built on first use per (chunk, quantum) and
// replayed by every later advance of the batch.
int chunk_graph(pfb_mr_batch *b, long long chunk, int quantum, cudaGraphExec_t *out) {
    for (const auto &g : b->graphs)
        if (g.chunk == chunk && g.quantum == quantum) {
            *out = g.exec;
            return PFB_OK;
        }
    JobDev *jobs = b->d_jobs;
    int n = b->n, q = quantum;
    int *locks = b->d_locks;
    unsigned int *counter = b->d_counter;
    const long long qpj = (chunk + quantum - 1) / quantum;
    unsigned int total = (unsigned int)std::min<long long>((long long)b->n * qpj, 0x7fffffffll);
    Twiddles tw = b->e->tw;
    void *args[] = {&jobs, &n, &locks, &counter, &total, &q, &tw};
    cudaGraph_t graph = nullptr;
    PFB_CUDA(cudaGraphCreate(&graph, 0));
    cudaMemsetParams mp{};
    mp.dst = counter;
    mp.value = 0;
    mp.elementSize = sizeof(unsigned int);
    mp.width = 1;
    mp.height = 1;
    cudaKernelNodeParams kp{};
    kp.func = (void *)persist_kernel;
    kp.gridDim = dim3((unsigned)std::min(b->n, std::max(1, b->e->num_sms)));
    kp.blockDim = dim3(THREADS);
    kp.sharedMemBytes = (unsigned)smem_bytes(b->maxlog);
    kp.kernelParams = args;
    cudaGraphNode_t n_mem = nullptr, n_ker = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaError_t ce = cudaGraphAddMemsetNode(&n_mem, graph, nullptr, 0, &mp);
    if (ce == cudaSuccess) ce = cudaGraphAddKernelNode(&n_ker, graph, &n_mem, 1, &kp);
    if (ce == cudaSuccess) ce = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) return pfb::cuda_fail(ce, "chunk graph", __FILE__, __LINE__);
    b->graphs.push_back(pfb_mr_batch::Graph{chunk, quantum, exec});
    *out = exec;
    return PFB_OK;
}

int batch_build(pfb_mr *e, const pfb_mr_number_t *nums, int n, uint32_t base, int mode,
                const pfb_mr_number_t *exps, pfb_mr_batch **out) {
    *out = nullptr;
    if (!e || !nums || n <= 0 || base < 2 || base > 0xFFFFu) {
        pfb::set_error("pfb_mr: bad argument (n=%d base=%u)", n, base);
        return PFB_E_ARG;
    }
    PFB_CUDA(cudaSetDevice(e->device));
    pfb_mr_batch *b = new pfb_mr_batch();
    b->e = e;
    b->n = n;
    b->mode = mode;
    prep_all(nums, n, base, mode, exps, b->hp);
    std::vector<Layout> lay(n);
    size_t total = 0;
    for (int i = 0; i < n; i++) {
        if (!b->hp[i].ok || b->hp[i].decided >= 0) continue;
        lay[i] = layout_for(b->hp[i], mode == 2);
        total += lay[i].total;
        b->maxlog = std::max(b->maxlog, b->hp[i].logl);
        b->max_steps = std::max(b->max_steps, (long long)b->hp[i].cursor + 2 + b->hp[i].s);
        b->n_ok++;
    }
    const size_t job_bytes = ((size_t)n * sizeof(JobDev) + 255) & ~(size_t)255;
    const size_t lock_bytes = ((size_t)n * sizeof(int) + 256 + 255) & ~(size_t)255;
    const size_t lucas_bytes = mode == 2 ? (((size_t)n * sizeof(LucasDev) + 255) & ~(size_t)255) : 0;
    const size_t need = job_bytes + lock_bytes + lucas_bytes + total * sizeof(uint32_t);
    if (cudaMalloc(&b->d_arena, need) != cudaSuccess) {
        cudaGetLastError();
        pfb::set_error("pfb_mr: cannot allocate %zu bytes of device memory", need);
        delete b;
        return PFB_E_NOMEM;
    }
    b->d_jobs = (JobDev *)b->d_arena;
    b->d_locks = (int *)(b->d_arena + job_bytes);
    b->d_counter = (unsigned int *)(b->d_arena + job_bytes + lock_bytes - 256);
    if (mode == 2) {
        b->d_lucas = (LucasDev *)(b->d_arena + job_bytes + lock_bytes);
        b->lucas.assign(n, LucasDev{});
    }
    uint32_t *d_words = (uint32_t *)(b->d_arena + job_bytes + lock_bytes + lucas_bytes);
    if (cudaMemsetAsync(b->d_locks, 0, lock_bytes, e->stream) != cudaSuccess) {
        batch_free(b);
        return pfb::cuda_fail(cudaGetLastError(), "lock reset", __FILE__, __LINE__);
    }
    b->jobs.assign(n, JobDev{});
    size_t off = 0;
    int rc = PFB_OK;
    for (int i = 0; i < n && !rc; i++) {
        JobDev &j = b->jobs[i];
        memset(&j, 0, sizeof(j));
        const HostPrep &h = b->hp[i];
        if (!h.ok || h.decided >= 0) {
            j.phase = 3;
            j.verdict = h.ok ? h.decided : -1;
            continue;
        }
        uint32_t *w = d_words + off;
        const Layout &l = lay[i];
        j.x = w + l.x;
        j.res = w + l.res;
        j.nn = w + l.nn;
        j.nh = w + l.nh;
        j.npl = w + l.npl;
        j.nl = w + l.nl;
        j.exp = w + l.exp;
        if (h.logl > LOG_LCTA) j.ybuf = w + l.yb;
        j.logl = h.logl;
        j.cursor = h.cursor;
        j.extra = mode >= 1 ? h.s - 1 : 0;
        j.phase = 0;
        j.base = base;
        j.mode = mode;
        const size_t H = h.x0.size();
        cudaError_t ce = cudaMemcpyAsync(j.x, h.x0.data(), H * 4, cudaMemcpyHostToDevice, e->stream);
        if (mode == 2) {
            LucasDev &lc = b->lucas[i];
            lc.lv0 = w + l.lv0;
            lc.lv1 = w + l.lv1;
            lc.lqk = w + l.lqk;
            lc.lt = w + l.lt;
            lc.lone = w + l.lone;
            lc.gy = w + l.gy;
            lc.q = h.q;
            lc.lb = h.lb;
            j.lucas = b->d_lucas + i;
            // V_0 = 2, V_1 = P = 1, Q^0 = 1, and 1 itself, in Montgomery form
            if (ce == cudaSuccess) ce = cudaMemcpyAsync(lc.lv0, h.v0.data(), H * 4, cudaMemcpyHostToDevice, e->stream);
            if (ce == cudaSuccess) ce = cudaMemcpyAsync(lc.lv1, h.x0.data(), H * 4, cudaMemcpyHostToDevice, e->stream);
            if (ce == cudaSuccess) ce = cudaMemcpyAsync(lc.lqk, h.x0.data(), H * 4, cudaMemcpyHostToDevice, e->stream);
            if (ce == cudaSuccess) ce = cudaMemcpyAsync(lc.lone, h.x0.data(), H * 4, cudaMemcpyHostToDevice, e->stream);
        }
        if (ce == cudaSuccess) ce = cudaMemcpyAsync((void *)j.npl, h.npl.data(), H * 4, cudaMemcpyHostToDevice, e->stream);
        if (ce == cudaSuccess) ce = cudaMemcpyAsync((void *)j.nl, h.nl.data(), H * 4, cudaMemcpyHostToDevice, e->stream);
        if (ce == cudaSuccess)
            ce = cudaMemcpyAsync((void *)j.exp, h.exp.data(), h.exp.size() * 4, cudaMemcpyHostToDevice, e->stream);
        if (ce != cudaSuccess) rc = pfb::cuda_fail(ce, "batch upload", __FILE__, __LINE__);
        off += l.total;
    }
    cudaError_t ce = cudaSuccess;
    if (!rc) ce = cudaMemcpyAsync(b->d_jobs, b->jobs.data(), n * sizeof(JobDev), cudaMemcpyHostToDevice, e->stream);
    if (!rc && ce == cudaSuccess && mode == 2)
        ce = cudaMemcpyAsync(b->d_lucas, b->lucas.data(), n * sizeof(LucasDev), cudaMemcpyHostToDevice, e->stream);
    if (!rc && ce != cudaSuccess) rc = pfb::cuda_fail(ce, "job upload", __FILE__, __LINE__);
    if (!rc && b->n_ok) {
        prep_kernel<<<n, THREADS, smem_bytes(b->maxlog), e->stream>>>(b->d_jobs, nullptr, e->tw);
        ce = cudaGetLastError();
        if (ce != cudaSuccess) rc = pfb::cuda_fail(ce, "prep_kernel", __FILE__, __LINE__);
    }
    // host staging must outlive the copies; later work may use other streams
    if (!rc) {
        ce = cudaStreamSynchronize(e->stream);
        if (ce != cudaSuccess) rc = pfb::cuda_fail(ce, "batch sync", __FILE__, __LINE__);
    }
    if (rc) {
        batch_free(b);
        return rc;
    }
    *out = b;
    return PFB_OK;
}

// Enqueues about `steps` steps of every unfinished candidate: launches of the
// persistent kernel, each handing out n * ceil(chunk / quantum) quanta.
int batch_advance(pfb_mr_batch *b, long long steps, cudaStream_t st) {
    if (!b->n_ok || steps <= 0) return PFB_OK;
    const long long cmax = b->e->chunk[b->maxlog];
    const int q0 = b->e->quantum[b->maxlog];
    while (steps > 0) {
        const long long chunk = std::min<long long>(steps, cmax);
        const int quantum = (int)std::min<long long>(chunk, q0);
        cudaGraphExec_t g = nullptr;
        const int rc = chunk_graph(b, chunk, quantum, &g);
        if (rc) return rc;
        PFB_CUDA(cudaGraphLaunch(g, st));
        steps -= chunk;
        b->steps_done += chunk;
    }
    return PFB_OK;
}

int batch_pending(pfb_mr_batch *b, int *pending, long long *steps_total) {
    PFB_CUDA(cudaStreamSynchronize(b->e->stream));
    PFB_CUDA(cudaDeviceSynchronize());
    PFB_CUDA(cudaMemcpy(b->jobs.data(), b->d_jobs, b->n * sizeof(JobDev), cudaMemcpyDeviceToHost));
    int c = 0;
    long long st = 0;
    for (int i = 0; i < b->n; i++) {
        c += b->jobs[i].phase != 3;
        st += b->jobs[i].steps;
    }
    if (pending) *pending = c;
    if (steps_total) *steps_total = st;
    return PFB_OK;
}

int batch_results(pfb_mr_batch *b, int8_t *verdict, uint16_t *residue, int residue_stride) {
    pfb_mr *e = b->e;
    PFB_CUDA(cudaMemcpyAsync(b->jobs.data(), b->d_jobs, b->n * sizeof(JobDev), cudaMemcpyDeviceToHost, e->stream));
    PFB_CUDA(cudaStreamSynchronize(e->stream));
    std::vector<uint32_t> r22;
    int rc = PFB_OK;
    for (int i = 0; i < b->n; i++) {
        const JobDev &j = b->jobs[i];
        if (!b->hp[i].ok || b->hp[i].decided >= 0) {
            if (verdict) verdict[i] = (int8_t)(b->hp[i].ok ? b->hp[i].decided : -1);
            if (residue) memset(residue + (size_t)i * residue_stride, 0, sizeof(uint16_t) * residue_stride);
            continue;
        }
        if (j.phase != 3) {
            if (verdict) verdict[i] = -2;
            rc = PFB_E_STATE;
            continue;
        }
        if (verdict) verdict[i] = (int8_t)(b->mode >= 1 ? j.verdict : 0);
        if (residue && b->mode != 2) {
            const size_t H = b->hp[i].x0.size();
            r22.resize(H);
            PFB_CUDA(cudaMemcpy(r22.data(), j.res, H * 4, cudaMemcpyDeviceToHost));
            pfb::big::Words r = pfb::big::from_limbs(r22.data(), LIMB_BITS, H);
            pfb::big::to_u16(r, residue + (size_t)i * residue_stride, (size_t)residue_stride);
        }
    }
    if (rc) pfb::set_error("pfb_mr: some candidates have not finished");
    return rc;
}

int run_jobs(pfb_mr *e, const pfb_mr_number_t *nums, int n, uint32_t base, int mode,
             const pfb_mr_number_t *exps, int8_t *verdict, uint16_t *residue, int residue_stride) {
    if (residue && residue_stride <= 0) {
        pfb::set_error("pfb_mr: residue_stride must be > 0");
        return PFB_E_ARG;
    }
    pfb_mr_batch *b = nullptr;
    int rc = batch_build(e, nums, n, base, mode, exps, &b);
    if (rc) return rc;
    rc = batch_advance(b, b->max_steps, e->stream);
    // The round-robin hands a locked candidate's quantum to another one, so a
    // few candidates may still need steps: continue until none is pending.
    // Every round advances each unfinished candidate, so a round count of
    // max_steps / 4096 + 64 is never reached unless the device stopped
    // making progress.
    const long long max_rounds = b->max_steps / 4096 + 64;
    for (long long round = 0; !rc; round++) {
        int pending = 0;
        rc = batch_pending(b, &pending, nullptr);
        if (rc || pending == 0) break;
        if (round >= max_rounds) {
            pfb::set_error("pfb_mr: %d candidates unfinished after %lld extra rounds", pending, round);
            rc = PFB_E_STATE;
            break;
        }
        rc = batch_advance(b, 4096, e->stream);
    }
    if (!rc) rc = batch_results(b, verdict, residue, residue_stride);
    cudaStreamSynchronize(e->stream);
    batch_free(b);
    return rc;
}

}  // namespace

extern "C" int pfb_mr_test(pfb_mr_t *e, const pfb_mr_number_t *nums, int n, uint32_t base, int8_t *verdict,
                           uint16_t *residue, int residue_stride) {
    return run_jobs(e, nums, n, base, 1, nullptr, verdict, residue, residue_stride);
}

extern "C" int pfb_mr_lucas(pfb_mr_t *e, const pfb_mr_number_t *nums, int n, int8_t *verdict) {
    if (!verdict) {
        pfb::set_error("pfb_mr_lucas: verdict is required");
        return PFB_E_ARG;
    }
    return run_jobs(e, nums, n, 2u, 2, nullptr, verdict, nullptr, 0);
}

extern "C" int pfb_mr_powm(pfb_mr_t *e, const pfb_mr_number_t *nums, int n, uint32_t base,
                           const pfb_mr_number_t *exps, uint16_t *residue, int residue_stride) {
    if (!exps || !residue) {
        pfb::set_error("pfb_mr_powm: exps and residue are required");
        return PFB_E_ARG;
    }
    return run_jobs(e, nums, n, base, 0, exps, nullptr, residue, residue_stride);
}

extern "C" int pfb_mr_batch_create(pfb_mr_t *e, const pfb_mr_number_t *nums, int n, uint32_t base,
                                   pfb_mr_batch_t **out) {
    if (!out) {
        pfb::set_error("pfb_mr_batch_create: null out");
        return PFB_E_ARG;
    }
    return batch_build(e, nums, n, base, 1, nullptr, out);
}

extern "C" int pfb_mr_batch_advance(pfb_mr_batch_t *b, int steps, void *stream) {
    if (!b || steps < 0) {
        pfb::set_error("pfb_mr_batch_advance: bad argument");
        return PFB_E_ARG;
    }
    PFB_CUDA(cudaSetDevice(b->e->device));
    return batch_advance(b, steps, stream ? (cudaStream_t)stream : b->e->stream);
}

extern "C" int pfb_mr_batch_pending(pfb_mr_batch_t *b, int *pending) {
    if (!b || !pending) {
        pfb::set_error("pfb_mr_batch_pending: bad argument");
        return PFB_E_ARG;
    }
    PFB_CUDA(cudaSetDevice(b->e->device));
    return batch_pending(b, pending, nullptr);
}

extern "C" long long pfb_mr_batch_steps_done(pfb_mr_batch_t *b) {
    if (!b) return -1;
    if (cudaSetDevice(b->e->device) != cudaSuccess) return -1;
    long long st = 0;
    if (batch_pending(b, nullptr, &st)) return -1;
    return st;
}

extern "C" long long pfb_mr_batch_steps_left(pfb_mr_batch_t *b) {
    if (!b) return -1;
    return std::max(0ll, b->max_steps - b->steps_done);
}

extern "C" int pfb_mr_batch_results(pfb_mr_batch_t *b, int8_t *verdict, uint16_t *residue, int residue_stride) {
    if (!b || (residue && residue_stride <= 0)) {
        pfb::set_error("pfb_mr_batch_results: bad argument");
        return PFB_E_ARG;
    }
    PFB_CUDA(cudaSetDevice(b->e->device));
    PFB_CUDA(cudaDeviceSynchronize());
    return batch_results(b, verdict, residue, residue_stride);
}

extern "C" void pfb_mr_batch_destroy(pfb_mr_batch_t *b) {
    if (!b) return;
    cudaSetDevice(b->e->device);
    cudaDeviceSynchronize();
    batch_free(b);
}

extern "C" int pfb_mr_autotune(pfb_mr_t *e, int logl_lo, int logl_hi, pfb_mr_tune_t *results, int cap,
                               int *n_results) {
    if (!e || logl_lo < LOG_LMIN || logl_hi > LOG_LSEQ || logl_lo > logl_hi || (cap > 0 && !results)) {
        pfb::set_error("pfb_mr_autotune: bad argument (transform lengths 2^%d .. 2^%d)", LOG_LMIN, LOG_LSEQ);
        return PFB_E_ARG;
    }
    if (n_results) *n_results = 0;
    PFB_CUDA(cudaSetDevice(e->device));
    // quanta above 64 steps leave SMs idle at the end of each launch once a
    // batch holds several candidates per SM, so the search stays below
    static const int kQuanta[] = {16, 32, 64};
    static const int kChunks[] = {1024, 2048};
    constexpr int NQ = 3, NC = 2, NP = NQ * NC;
    const long long kSteps = 2048;  // timed steps per tried pair and batch shape
    const int sms = std::max(1, e->num_sms);
    int rows = 0;
    uint64_t x = 0x9E3779B97F4A7C15ull;  // xorshift64: synthetic moduli
    cudaEvent_t ev[2];
    PFB_CUDA(cudaEventCreate(&ev[0]));
    PFB_CUDA(cudaEventCreate(&ev[1]));
    int rc = PFB_OK;
    for (int lg = logl_lo; lg <= logl_hi && !rc; lg++) {
        // the longest base-2 modulus of this length: R = 2^(22 L/2) >= 2^(bits + 6)
        const size_t bits = std::min<size_t>((size_t)LIMB_BITS * ((size_t)1 << (lg - 1)) - 8, PFB_MR_MAX_BITS);
        const int n16 = (int)((bits + 15) / 16);
        const int q_old = e->quantum[lg], c_old = e->chunk[lg];
        double rate[2][NP] = {};
        // two batch shapes: one and two candidates per SM (the tail of a launch
        // weighs more with one)
        for (int shape = 0; shape < 2 && !rc; shape++) {
            const int n = (shape + 1) * sms;
            std::vector<uint16_t> limbs((size_t)n * n16);
            std::vector<pfb_mr_number_t> nums(n);
            for (int i = 0; i < n; i++) {
                uint16_t *l = limbs.data() + (size_t)i * n16;
                for (int w = 0; w < n16; w++) {
                    x ^= x << 13;
                    x ^= x >> 7;
                    x ^= x << 17;
                    l[w] = (uint16_t)x;
                }
                const int top = (int)((bits - 1) % 16);
                l[n16 - 1] = (uint16_t)((l[n16 - 1] & ((1u << top) - 1u)) | (1u << top));
                l[0] |= 1u;
                nums[i] = pfb_mr_number_t{l, n16};
            }
            pfb_mr_batch *b = nullptr;
            rc = batch_build(e, nums.data(), n, 2u, 1, nullptr, &b);
            if (rc) break;
            rc = batch_advance(b, 64, e->stream);  // warm-up
            for (int k = 0; k < NP && !rc; k++) {
                e->quantum[lg] = kQuanta[k / NC];
                e->chunk[lg] = kChunks[k % NC];
                long long before = 0, after = 0;
                rc = batch_pending(b, nullptr, &before);
                if (!rc && cudaEventRecord(ev[0], e->stream) != cudaSuccess) rc = PFB_E_CUDA;
                if (!rc) rc = batch_advance(b, kSteps, e->stream);
                if (!rc && cudaEventRecord(ev[1], e->stream) != cudaSuccess) rc = PFB_E_CUDA;
                if (!rc) rc = batch_pending(b, nullptr, &after);
                float ms = 0.f;
                if (!rc && cudaEventElapsedTime(&ms, ev[0], ev[1]) != cudaSuccess) rc = PFB_E_CUDA;
                if (!rc) rate[shape][k] = ms > 0.f ? (double)(after - before) / (1e-3 * (double)ms) : 0.0;
            }
            batch_free(b);
        }
        e->quantum[lg] = q_old;
        e->chunk[lg] = c_old;
        if (rc) break;
        // score: the sum over shapes of the rate relative to the shape's best
        double best_rate[2] = {0.0, 0.0}, best = -1.0;
        for (int shape = 0; shape < 2; shape++)
            for (int k = 0; k < NP; k++) best_rate[shape] = std::max(best_rate[shape], rate[shape][k]);
        for (int k = 0; k < NP; k++) {
            double score = 0.0;
            for (int shape = 0; shape < 2; shape++)
                score += best_rate[shape] > 0.0 ? rate[shape][k] / best_rate[shape] : 0.0;
            if (results && rows < cap)
                results[rows] = pfb_mr_tune_t{lg, kQuanta[k / NC], kChunks[k % NC], rate[0][k], rate[1][k]};
            rows++;
            if (score > best) {
                best = score;
                e->quantum[lg] = kQuanta[k / NC];
                e->chunk[lg] = kChunks[k % NC];
            }
        }
    }
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    if (n_results) *n_results = std::min(rows, cap);
    return rc;
}

extern "C" int pfb_mr_get_tuning(pfb_mr_t *e, int logl, int *quantum, int *chunk) {
    if (!e || logl < 0 || logl > LOG_LMAX) {
        pfb::set_error("pfb_mr_get_tuning: bad argument");
        return PFB_E_ARG;
    }
    if (quantum) *quantum = e->quantum[logl];
    if (chunk) *chunk = e->chunk[logl];
    return PFB_OK;
}

extern "C" long long pfb_mr_test_cost(const uint16_t *limbs, int n_limbs) {
    if (!limbs || n_limbs <= 0) return -1;
    pfb::big::Words N = pfb::big::from_u16(limbs, (size_t)n_limbs);
    const size_t nb = pfb::big::bit_length(N);
    if (nb < 2) return -1;
    return (long long)nb;  // ~ bits(d) squarings + one conversion
}

// ===========================================================================
// Serving: continuous batching on one GPU.
//
// Requests (candidates of any length) are prepared on host worker threads
// (N', R mod N, exponent) and admitted into free slots of a device-resident
// job table between launches of the persistent kernel, as slots and the HBM
// budget allow; every launch advances all resident candidates, whatever
// their lengths, round-robin by quanta; finished candidates are retired with
// their timestamps and their slot memory returns to a size-class pool.  All
// host waits are bounded (condition variables with timeouts); nothing on the
// device waits.

#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>

namespace {

using Clock = std::chrono::steady_clock;

struct SrvRequest {
    uint64_t tag = 0;
    std::vector<uint16_t> limbs;
    uint16_t *residue_out = nullptr;
    int residue_cap = 0;
    double t_submit = 0.0, t_admit = 0.0;
    HostPrep hp;
};

struct SrvSlot {
    bool busy = false;
    int logl = 0;
    uint8_t *mem = nullptr;
    SrvRequest req;
};

}  // namespace

struct pfb_mr_server {
    pfb_mr *e = nullptr;
    pfb_mr_server_config_t cfg{};
    Clock::time_point t0;
    // device job table
    JobDev *d_jobs = nullptr;
    int *d_locks = nullptr;
    unsigned int *d_counter = nullptr;
    int *d_list = nullptr;
    uint8_t *d_table_mem = nullptr;
    std::vector<JobDev> jobs;
    std::vector<SrvSlot> slots;
    std::map<int, std::vector<uint8_t *>> pool;  // free slot memory by transform length
    size_t bytes_in_use = 0, bytes_owned = 0;
    cudaStream_t stream = nullptr;
    // queues
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<SrvRequest> submitted, prepared;
    std::deque<pfb_mr_result_t> done;
    bool stop = false;
    int preparing = 0;
    // statistics
    long long n_submitted = 0, n_admitted = 0, n_completed = 0, launches = 0;
    long long steps_total = 0;
    int resident = 0;
    std::vector<std::thread> workers;
    std::thread driver;
    int error = PFB_OK;
    // host-side fault injection (pfb_mr_server_inject_alloc_failures)
    int inject_alloc_failures = 0;
    int injected_alloc_failures = 0;
};

namespace {

double now_s(const pfb_mr_server *s) {
    return std::chrono::duration<double>(Clock::now() - s->t0).count();
}

size_t slot_bytes(int logl) { return slot_layout(logl).total * sizeof(uint32_t); }

// Slot memory; a failure injected from the host (a test hook) is reported as
// cudaErrorMemoryAllocation without calling cudaMalloc.
cudaError_t srv_alloc(pfb_mr_server *s, uint8_t **mem, size_t need) {
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->inject_alloc_failures > 0) {
            s->inject_alloc_failures--;
            s->injected_alloc_failures++;
            return cudaErrorMemoryAllocation;
        }
    }
    return cudaMalloc(mem, need);
}

void srv_prep_worker(pfb_mr_server *s) {
    for (;;) {
        SrvRequest r;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            while (!s->stop && s->submitted.empty()) s->cv_work.wait_for(lk, std::chrono::milliseconds(100));
            if (s->stop) return;
            r = std::move(s->submitted.front());
            s->submitted.pop_front();
            s->preparing++;
        }
        pfb_mr_number_t num{r.limbs.data(), (int)r.limbs.size()};
        host_prep(num, s->cfg.base, 1, nullptr, r.hp);
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->preparing--;
            if (!r.hp.ok) {
                pfb_mr_result_t res{};
                res.tag = r.tag;
                res.verdict = -1;
                res.submit_s = r.t_submit;
                res.admit_s = res.done_s = now_s(s);
                s->done.push_back(res);
                s->n_completed++;
                s->cv_done.notify_all();
            } else {
                s->prepared.push_back(std::move(r));
            }
        }
        s->cv_work.notify_all();
    }
}

// Admits prepared requests into free slots; returns the slots admitted.
int srv_admit(pfb_mr_server *s, std::vector<int> &admitted) {
    admitted.clear();
    for (;;) {
        SrvRequest r;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            if (s->prepared.empty()) break;
            int free_slot = -1;
            for (int i = 0; i < (int)s->slots.size(); i++)
                if (!s->slots[i].busy) {
                    free_slot = i;
                    break;
                }
            if (free_slot < 0) break;
            const int lg = s->prepared.front().hp.logl;
            const size_t need = slot_bytes(lg);
            const bool pooled = !s->pool[lg].empty();
            if (s->cfg.hbm_budget_bytes && !pooled && s->bytes_owned + need > s->cfg.hbm_budget_bytes) {
                // give back pooled blocks of other lengths first
                for (auto &kv : s->pool) {
                    while (!kv.second.empty() && s->bytes_owned + need > s->cfg.hbm_budget_bytes) {
                        const size_t blk = slot_bytes(kv.first);
                        cudaFree(kv.second.back());
                        kv.second.pop_back();
                        s->bytes_owned -= std::min(s->bytes_owned, blk);
                    }
                }
            }
            if (s->cfg.hbm_budget_bytes && !pooled && s->bytes_owned + need > s->cfg.hbm_budget_bytes) {
                if (s->resident == 0 && admitted.empty()) {
                    // a single request above the whole budget can never run
                    SrvRequest bad = std::move(s->prepared.front());
                    s->prepared.pop_front();
                    pfb_mr_result_t res{};
                    res.tag = bad.tag;
                    res.verdict = -1;
                    res.submit_s = bad.t_submit;
                    res.admit_s = res.done_s = now_s(s);
                    s->done.push_back(res);
                    s->n_completed++;
                    s->cv_done.notify_all();
                    continue;
                }
                break;  // wait for memory to come back
            }
            r = std::move(s->prepared.front());
            s->prepared.pop_front();
            SrvSlot &sl = s->slots[free_slot];
            sl.busy = true;
            sl.logl = lg;
            if (pooled) {
                sl.mem = s->pool[lg].back();
                s->pool[lg].pop_back();
            } else {
                sl.mem = nullptr;
            }
            s->bytes_in_use += need;
            admitted.push_back(free_slot);
            r.t_admit = now_s(s);
            sl.req = std::move(r);
        }
        SrvSlot &sl = s->slots[admitted.back()];
        if (!sl.mem) {
            const size_t need = slot_bytes(sl.logl);
            cudaError_t ce = srv_alloc(s, &sl.mem, need);
            if (ce != cudaSuccess) {
                // the device ran out below the budget (memory held elsewhere):
                // give back the pooled blocks and try once more
                cudaGetLastError();
                std::lock_guard<std::mutex> lk(s->mu);
                for (auto &kv : s->pool) {
                    const size_t blk = slot_bytes(kv.first);
                    for (uint8_t *m : kv.second) {
                        cudaFree(m);
                        s->bytes_owned -= std::min(s->bytes_owned, blk);
                    }
                    kv.second.clear();
                }
                sl.mem = nullptr;
            }
            if (ce != cudaSuccess) ce = srv_alloc(s, &sl.mem, need);
            if (ce != cudaSuccess) {
                // undo the admission: the request waits for resident candidates
                // to retire, or fails if none is resident
                cudaGetLastError();
                sl.mem = nullptr;
                admitted.pop_back();
                std::lock_guard<std::mutex> lk(s->mu);
                sl.busy = false;
                s->bytes_in_use -= need;
                if (s->resident == 0 && admitted.empty()) {
                    pfb_mr_result_t res{};
                    res.tag = sl.req.tag;
                    res.verdict = -1;
                    res.submit_s = sl.req.t_submit;
                    res.admit_s = res.done_s = now_s(s);
                    s->done.push_back(res);
                    s->n_completed++;
                    s->cv_done.notify_all();
                } else {
                    s->prepared.push_front(std::move(sl.req));
                }
                sl.req = SrvRequest();
                break;
            }
            std::lock_guard<std::mutex> lk(s->mu);
            s->bytes_owned += need;
        }
        // fill the job and upload its inputs
        const HostPrep &h = sl.req.hp;
        const Layout l = slot_layout(h.logl);
        uint32_t *w = (uint32_t *)sl.mem;
        JobDev &j = s->jobs[admitted.back()];
        memset(&j, 0, sizeof(j));
        j.x = w + l.x;
        j.res = w + l.res;
        j.nn = w + l.nn;
        j.nh = w + l.nh;
        j.npl = w + l.npl;
        j.nl = w + l.nl;
        j.exp = w + l.exp;
        if (h.logl > LOG_LCTA) j.ybuf = w + l.yb;
        j.logl = h.logl;
        j.cursor = h.cursor;
        j.extra = h.s - 1;
        j.phase = 0;
        j.base = s->cfg.base;
        j.mode = 1;
        const size_t H = h.x0.size();
        PFB_CUDA(cudaMemcpyAsync(j.x, h.x0.data(), H * 4, cudaMemcpyHostToDevice, s->stream));
        PFB_CUDA(cudaMemcpyAsync((void *)j.npl, h.npl.data(), H * 4, cudaMemcpyHostToDevice, s->stream));
        PFB_CUDA(cudaMemcpyAsync((void *)j.nl, h.nl.data(), H * 4, cudaMemcpyHostToDevice, s->stream));
        PFB_CUDA(cudaMemcpyAsync((void *)j.exp, h.exp.data(), h.exp.size() * 4, cudaMemcpyHostToDevice, s->stream));
        PFB_CUDA(cudaMemcpyAsync(s->d_jobs + admitted.back(), &j, sizeof(JobDev), cudaMemcpyHostToDevice, s->stream));
        PFB_CUDA(cudaStreamSynchronize(s->stream));  // host staging is freed below / reused
    }
    if (!admitted.empty()) {
        PFB_CUDA(cudaMemcpyAsync(s->d_list, admitted.data(), admitted.size() * sizeof(int), cudaMemcpyHostToDevice,
                                 s->stream));
        int maxlog = LOG_LMIN;
        for (int i : admitted) maxlog = std::max(maxlog, s->slots[i].logl);
        prep_kernel<<<(int)admitted.size(), THREADS, smem_bytes(maxlog), s->stream>>>(s->d_jobs, s->d_list, s->e->tw);
        PFB_CUDA(cudaGetLastError());
        PFB_CUDA(cudaStreamSynchronize(s->stream));
        for (int i : admitted) {  // the set-up inputs are on the device now
            HostPrep &h = s->slots[i].req.hp;
            std::vector<uint32_t>().swap(h.npl);
            std::vector<uint32_t>().swap(h.exp);
        }
        std::lock_guard<std::mutex> lk(s->mu);
        s->resident += (int)admitted.size();
        s->n_admitted += (long long)admitted.size();
    }
    return PFB_OK;
}

// Retires finished candidates (host mirror of the job table already read).
void srv_retire(pfb_mr_server *s) {
    std::vector<uint32_t> r22;
    for (int i = 0; i < (int)s->slots.size(); i++) {
        SrvSlot &sl = s->slots[i];
        if (!sl.busy || s->jobs[i].phase != 3) continue;
        pfb_mr_result_t res{};
        res.tag = sl.req.tag;
        res.verdict = (int8_t)s->jobs[i].verdict;
        res.submit_s = sl.req.t_submit;
        res.admit_s = sl.req.t_admit;
        if (sl.req.residue_out && sl.req.residue_cap > 0) {
            const size_t H = sl.req.hp.x0.size();
            r22.resize(H);
            if (cudaMemcpy(r22.data(), s->jobs[i].res, H * 4, cudaMemcpyDeviceToHost) == cudaSuccess) {
                pfb::big::Words r = pfb::big::from_limbs(r22.data(), LIMB_BITS, H);
                pfb::big::to_u16(r, sl.req.residue_out, (size_t)sl.req.residue_cap);
            }
        }
        res.done_s = now_s(s);
        const size_t bytes = slot_bytes(sl.logl);
        std::lock_guard<std::mutex> lk(s->mu);
        s->pool[sl.logl].push_back(sl.mem);
        sl.mem = nullptr;
        sl.busy = false;
        s->bytes_in_use -= bytes;
        s->resident--;
        s->n_completed++;
        s->steps_total += s->jobs[i].steps;
        s->done.push_back(res);
        s->cv_done.notify_all();
    }
}

void srv_driver(pfb_mr_server *s) {
    if (cudaSetDevice(s->e->device) != cudaSuccess) {
        s->error = PFB_E_CUDA;
        return;
    }
    std::vector<int> admitted;
    const int cap = (int)s->slots.size();
    const int grid_max = std::max(1, s->e->num_sms);
    while (true) {
        {
            std::unique_lock<std::mutex> lk(s->mu);
            while (!s->stop && s->resident == 0 && s->prepared.empty())
                s->cv_work.wait_for(lk, std::chrono::milliseconds(50));
            if (s->stop) break;
        }
        int rc = srv_admit(s, admitted);
        if (rc) {
            s->error = rc;
            break;
        }
        int res_now;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            res_now = s->resident;
        }
        if (res_now == 0) continue;
        // one launch: every resident candidate advances about chunk_steps steps
        const int quantum = std::min(64, s->cfg.chunk_steps);
        const long long qpj = (s->cfg.chunk_steps + quantum - 1) / quantum;
        int maxlog = LOG_LMIN;
        for (auto &sl : s->slots)
            if (sl.busy) maxlog = std::max(maxlog, sl.logl);
        cudaMemsetAsync(s->d_counter, 0, sizeof(unsigned int), s->stream);
        persist_kernel<<<std::min(res_now, grid_max), THREADS, smem_bytes(maxlog), s->stream>>>(
            s->d_jobs, cap, s->d_locks, s->d_counter, (unsigned int)(res_now * qpj), quantum, s->e->tw);
        if (cudaGetLastError() != cudaSuccess ||
            cudaMemcpyAsync(s->jobs.data(), s->d_jobs, cap * sizeof(JobDev), cudaMemcpyDeviceToHost, s->stream) !=
                cudaSuccess ||
            cudaStreamSynchronize(s->stream) != cudaSuccess) {
            pfb::set_error("pfb_mr_server: CUDA failure in the step loop");
            s->error = PFB_E_CUDA;
            break;
        }
        s->launches++;
        srv_retire(s);
    }
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    s->cv_done.notify_all();
    s->cv_work.notify_all();
}

}  // namespace

extern "C" int pfb_mr_server_create(pfb_mr_t *e, const pfb_mr_server_config_t *cfg, pfb_mr_server_t **out) {
    if (!e || !out) {
        pfb::set_error("pfb_mr_server_create: null argument");
        return PFB_E_ARG;
    }
    *out = nullptr;
    pfb_mr_server *s = new pfb_mr_server();
    s->e = e;
    if (cfg) s->cfg = *cfg;
    if (s->cfg.max_resident <= 0) s->cfg.max_resident = 2 * std::max(1, e->num_sms);
    if (s->cfg.chunk_steps <= 0) s->cfg.chunk_steps = 512;
    if (s->cfg.base < 2 || s->cfg.base > 0xFFFFu) s->cfg.base = 2;
    if (s->cfg.prep_threads <= 0) s->cfg.prep_threads = 4;
    s->t0 = Clock::now();
    const int cap = s->cfg.max_resident;
    PFB_CUDA(cudaSetDevice(e->device));
    const size_t job_bytes = ((size_t)cap * sizeof(JobDev) + 255) & ~(size_t)255;
    const size_t int_bytes = ((size_t)cap * sizeof(int) + 255) & ~(size_t)255;
    if (cudaMalloc(&s->d_table_mem, job_bytes + 2 * int_bytes + 256) != cudaSuccess) {
        cudaGetLastError();
        delete s;
        pfb::set_error("pfb_mr_server_create: cannot allocate the job table");
        return PFB_E_NOMEM;
    }
    s->d_jobs = (JobDev *)s->d_table_mem;
    s->d_locks = (int *)(s->d_table_mem + job_bytes);
    s->d_list = (int *)(s->d_table_mem + job_bytes + int_bytes);
    s->d_counter = (unsigned int *)(s->d_table_mem + job_bytes + 2 * int_bytes);
    s->jobs.assign(cap, JobDev{});
    for (auto &j : s->jobs) j.phase = 3;
    s->slots.resize(cap);
    int rc = PFB_OK;
    cudaError_t ce = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (ce == cudaSuccess) ce = cudaMemcpy(s->d_jobs, s->jobs.data(), cap * sizeof(JobDev), cudaMemcpyHostToDevice);
    if (ce == cudaSuccess) ce = cudaMemset(s->d_locks, 0, int_bytes);
    if (ce != cudaSuccess) rc = pfb::cuda_fail(ce, "server set-up", __FILE__, __LINE__);
    if (rc) {
        cudaFree(s->d_table_mem);
        if (s->stream) cudaStreamDestroy(s->stream);
        delete s;
        return rc;
    }
    for (int t = 0; t < s->cfg.prep_threads; t++) s->workers.emplace_back(srv_prep_worker, s);
    s->driver = std::thread(srv_driver, s);
    *out = s;
    return PFB_OK;
}

extern "C" int pfb_mr_server_submit(pfb_mr_server_t *s, const uint16_t *limbs, int n_limbs, uint64_t tag,
                                    uint16_t *residue_out, int residue_cap) {
    if (!s || !limbs || n_limbs <= 0 || (residue_out && residue_cap <= 0)) {
        pfb::set_error("pfb_mr_server_submit: bad argument");
        return PFB_E_ARG;
    }
    SrvRequest r;
    r.tag = tag;
    r.limbs.assign(limbs, limbs + n_limbs);
    r.residue_out = residue_out;
    r.residue_cap = residue_cap;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) {
            pfb::set_error("pfb_mr_server_submit: server stopped (%d)", s->error);
            return PFB_E_STATE;
        }
        r.t_submit = now_s(s);
        s->submitted.push_back(std::move(r));
        s->n_submitted++;
    }
    s->cv_work.notify_all();
    return PFB_OK;
}

extern "C" int pfb_mr_server_poll(pfb_mr_server_t *s, pfb_mr_result_t *out, int cap, int timeout_ms) {
    if (!s || !out || cap <= 0) {
        pfb::set_error("pfb_mr_server_poll: bad argument");
        return PFB_E_ARG;
    }
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->done.empty() && timeout_ms > 0 && !s->stop)
        s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return !s->done.empty() || s->stop; });
    int n = 0;
    while (n < cap && !s->done.empty()) {
        out[n++] = s->done.front();
        s->done.pop_front();
    }
    if (n == 0 && s->stop && s->error) return s->error;
    return n;
}

extern "C" int pfb_mr_server_inject_alloc_failures(pfb_mr_server_t *s, int n) {
    if (!s || n < 0) {
        pfb::set_error("pfb_mr_server_inject_alloc_failures: bad argument");
        return PFB_E_ARG;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    s->inject_alloc_failures += n;
    return s->injected_alloc_failures;
}

extern "C" int pfb_mr_server_stats(pfb_mr_server_t *s, pfb_mr_server_stats_t *st) {
    if (!s || !st) {
        pfb::set_error("pfb_mr_server_stats: bad argument");
        return PFB_E_ARG;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    st->submitted = s->n_submitted;
    st->admitted = s->n_admitted;
    st->completed = s->n_completed;
    st->resident = s->resident;
    st->queued = (int)(s->submitted.size() + s->prepared.size()) + s->preparing;
    st->launches = s->launches;
    st->steps_retired = s->steps_total;
    st->bytes_in_use = s->bytes_in_use;
    st->bytes_owned = s->bytes_owned;
    st->error = s->error;
    return PFB_OK;
}

extern "C" void pfb_mr_server_destroy(pfb_mr_server_t *s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    s->cv_done.notify_all();
    if (s->driver.joinable()) s->driver.join();
    for (auto &t : s->workers)
        if (t.joinable()) t.join();
    cudaSetDevice(s->e->device);
    cudaStreamSynchronize(s->stream);
    for (auto &sl : s->slots)
        if (sl.mem) cudaFree(sl.mem);
    for (auto &kv : s->pool)
        for (uint8_t *m : kv.second) cudaFree(m);
    cudaFree(s->d_table_mem);
    cudaStreamDestroy(s->stream);
    delete s;
}

// ---------------------------------------------------------------------------
// Per-operation modular context (BatchModCtx's methods).

struct pfb_mr_ctx {
    pfb_mr *e = nullptr;
    int n = 0, n16 = 0, maxlog = LOG_LMIN;
    uint8_t *d_arena = nullptr;
    JobDev *d_jobs = nullptr;
    CtxExtra *d_ex = nullptr;
    uint64_t *d_one = nullptr, *d_nm1 = nullptr, *d_tmp = nullptr, *d_n = nullptr;  // [n][n16] each
    std::vector<HostPrep> hp;
};

namespace {

int ctx_fail(pfb_mr_ctx *c, int rc) {
    if (c) {
        cudaFree(c->d_arena);
        delete c;
    }
    return rc;
}

std::vector<uint64_t> widen16(const pfb::big::Words &w, size_t n16) {
    std::vector<uint16_t> t(n16);
    pfb::big::to_u16(w, t.data(), n16);
    return std::vector<uint64_t>(t.begin(), t.end());
}

int ctx_launch(pfb_mr_ctx *c, const uint64_t *a, const uint64_t *b, uint64_t *out, int out_stride, int op,
               void *stream) {
    if (!c || !a || !out || ((op == CTX_MODMUL || op == CTX_RAW_MUL) && !b)) {
        pfb::set_error("pfb_mr_ctx: bad argument");
        return PFB_E_ARG;
    }
    PFB_CUDA(cudaSetDevice(c->e->device));
    // NULL: the legacy default stream, ordered with the caller's other
    // default-stream work (the reference's methods run there)
    cudaStream_t st = stream ? (cudaStream_t)stream : cudaStreamLegacy;
    ctx_kernel<<<c->n, THREADS, smem_bytes(c->maxlog), st>>>(c->d_jobs, c->d_ex, a, b ? b : a, out, c->n16,
                                                              out_stride, op, c->e->tw);
    PFB_CUDA(cudaGetLastError());
    return PFB_OK;
}

}  // namespace

extern "C" int pfb_mr_ctx_create(pfb_mr_t *e, const uint64_t *N_all, int n_limbs, int n_batch, pfb_mr_ctx_t **out) {
    if (!out || !e || !N_all || n_limbs <= 0 || n_batch <= 0) {
        pfb::set_error("pfb_mr_ctx_create: bad argument");
        return PFB_E_ARG;
    }
    *out = nullptr;
    PFB_CUDA(cudaSetDevice(e->device));
    pfb_mr_ctx *c = new pfb_mr_ctx();
    c->e = e;
    c->n = n_batch;
    c->n16 = n_limbs;
    std::vector<uint16_t> n16((size_t)n_limbs * n_batch);
    for (size_t i = 0; i < n16.size(); i++) {
        if (N_all[i] > 0xFFFFu) {
            pfb::set_error("pfb_mr_ctx_create: limb %zu is not a 16-bit value", i);
            return ctx_fail(c, PFB_E_ARG);
        }
        n16[i] = (uint16_t)N_all[i];
    }
    std::vector<pfb_mr_number_t> nums(n_batch);
    for (int i = 0; i < n_batch; i++) nums[i] = pfb_mr_number_t{n16.data() + (size_t)i * n_limbs, n_limbs};
    // base 2 sizes R > 64 N: products of two reduced operands stay below 2N after REDC
    prep_all(nums.data(), n_batch, 2u, 1, nullptr, c->hp);
    std::vector<Layout> lay(n_batch);
    size_t words = 0;
    for (int i = 0; i < n_batch; i++) {
        if (!c->hp[i].ok) {
            pfb::set_error("pfb_mr_ctx_create: modulus %d is not odd, > 1 and at most %d bits", i, PFB_MR_MAX_BITS);
            return ctx_fail(c, PFB_E_ARG);
        }
        lay[i] = layout_for(c->hp[i].logl, 1, true, true);  // gy [2][L], spare H-word buffers, raw coefficients
        words += lay[i].total;
        c->maxlog = std::max(c->maxlog, c->hp[i].logl);
    }
    const size_t job_bytes = ((size_t)n_batch * sizeof(JobDev) + 255) & ~(size_t)255;
    const size_t ex_bytes = ((size_t)n_batch * sizeof(CtxExtra) + 255) & ~(size_t)255;
    const size_t v_bytes = (((size_t)n_batch * n_limbs * sizeof(uint64_t)) + 255) & ~(size_t)255;
    const size_t need = job_bytes + ex_bytes + 4 * v_bytes + words * sizeof(uint32_t);
    if (cudaMalloc(&c->d_arena, need) != cudaSuccess) {
        cudaGetLastError();
        pfb::set_error("pfb_mr_ctx_create: cannot allocate %zu bytes of device memory", need);
        return ctx_fail(c, PFB_E_NOMEM);
    }
    c->d_jobs = (JobDev *)c->d_arena;
    c->d_ex = (CtxExtra *)(c->d_arena + job_bytes);
    c->d_one = (uint64_t *)(c->d_arena + job_bytes + ex_bytes);
    c->d_nm1 = (uint64_t *)(c->d_arena + job_bytes + ex_bytes + v_bytes);
    c->d_tmp = (uint64_t *)(c->d_arena + job_bytes + ex_bytes + 2 * v_bytes);
    c->d_n = (uint64_t *)(c->d_arena + job_bytes + ex_bytes + 3 * v_bytes);
    uint32_t *d_words = (uint32_t *)(c->d_arena + job_bytes + ex_bytes + 4 * v_bytes);
    std::vector<JobDev> jobs(n_batch);
    std::vector<CtxExtra> ex(n_batch);
    std::vector<uint64_t> one((size_t)n_batch * n_limbs), nm1((size_t)n_batch * n_limbs);
    size_t off = 0;
    for (int i = 0; i < n_batch; i++) {
        const HostPrep &h = c->hp[i];
        const Layout &l = lay[i];
        uint32_t *w = d_words + off;
        JobDev &j = jobs[i];
        memset(&j, 0, sizeof(j));
        j.nn = w + l.nn;
        j.nh = w + l.nh;
        j.npl = w + l.npl;
        j.nl = w + l.nl;
        j.x = w + l.x;
        j.res = w + l.res;
        if (h.logl > LOG_LCTA) j.ybuf = w + l.yb;
        j.logl = h.logl;
        j.phase = 0;
        ex[i].gy = w + l.gy;
        ex[i].yl = w + l.lt;
        ex[i].raw = (unsigned long long *)(w + l.raw);
        const size_t H = h.nl.size();
        PFB_CUDA(cudaMemcpy((void *)j.npl, h.npl.data(), H * 4, cudaMemcpyHostToDevice));
        PFB_CUDA(cudaMemcpy((void *)j.nl, h.nl.data(), H * 4, cudaMemcpyHostToDevice));
        // working forms of 1 and N - 1: R mod N and N - (R mod N)
        const pfb::big::Words N = pfb::big::from_u16(nums[i].limbs, (size_t)n_limbs);
        const pfb::big::Words r = pfb::big::from_limbs(h.x0.data(), LIMB_BITS, H);
        const std::vector<uint64_t> o = widen16(r, (size_t)n_limbs), m = widen16(pfb::big::sub(N, r), (size_t)n_limbs);
        std::copy(o.begin(), o.end(), one.begin() + (size_t)i * n_limbs);
        std::copy(m.begin(), m.end(), nm1.begin() + (size_t)i * n_limbs);
        off += l.total;
    }
    PFB_CUDA(cudaMemcpy(c->d_jobs, jobs.data(), n_batch * sizeof(JobDev), cudaMemcpyHostToDevice));
    PFB_CUDA(cudaMemcpy(c->d_ex, ex.data(), n_batch * sizeof(CtxExtra), cudaMemcpyHostToDevice));
    PFB_CUDA(cudaMemcpy(c->d_one, one.data(), one.size() * 8, cudaMemcpyHostToDevice));
    PFB_CUDA(cudaMemcpy(c->d_nm1, nm1.data(), nm1.size() * 8, cudaMemcpyHostToDevice));
    const std::vector<uint64_t> nall(n16.begin(), n16.end());
    PFB_CUDA(cudaMemcpy(c->d_n, nall.data(), nall.size() * 8, cudaMemcpyHostToDevice));
    prep_kernel<<<n_batch, THREADS, smem_bytes(c->maxlog), e->stream>>>(c->d_jobs, nullptr, e->tw);
    cudaError_t ce = cudaGetLastError();
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    if (ce != cudaSuccess) return ctx_fail(c, pfb::cuda_fail(ce, "pfb_mr_ctx_create", __FILE__, __LINE__));
    *out = c;
    return PFB_OK;
}

extern "C" void pfb_mr_ctx_destroy(pfb_mr_ctx_t *c) {
    if (!c) return;
    cudaSetDevice(c->e->device);
    cudaDeviceSynchronize();
    ctx_fail(c, PFB_OK);
}

extern "C" int pfb_mr_ctx_n_sum(const pfb_mr_ctx_t *c) { return c ? 2 * c->n16 + 16 : -1; }

extern "C" int pfb_mr_ctx_buffers(const pfb_mr_ctx_t *c, const uint64_t **d_N, const uint64_t **d_one,
                                  const uint64_t **d_nm1) {
    if (!c) {
        pfb::set_error("pfb_mr_ctx_buffers: null context");
        return PFB_E_ARG;
    }
    if (d_N) *d_N = c->d_n;
    if (d_one) *d_one = c->d_one;
    if (d_nm1) *d_nm1 = c->d_nm1;
    return PFB_OK;
}

extern "C" int pfb_mr_ctx_to_residue(pfb_mr_ctx_t *c, const uint64_t *x_all, uint64_t *out_all) {
    if (!c || !x_all || !out_all) {
        pfb::set_error("pfb_mr_ctx_to_residue: bad argument");
        return PFB_E_ARG;
    }
    using namespace pfb::big;
    std::vector<uint16_t> t(c->n16);
    for (int i = 0; i < c->n; i++) {
        const size_t o = (size_t)i * c->n16;
        for (int k = 0; k < c->n16; k++) t[k] = (uint16_t)x_all[o + k];
        const Words x = from_u16(t.data(), (size_t)c->n16);
        const HostPrep &h = c->hp[i];
        const Words N = from_limbs(h.nl.data(), LIMB_BITS, h.nl.size());
        Words rem;
        divmod(add(shl(x, (size_t)LIMB_BITS * h.nl.size()), x), N, nullptr, &rem);  // x R' mod N, R' = 2^(22 H) + 1
        const std::vector<uint64_t> r = widen16(rem, (size_t)c->n16);
        std::copy(r.begin(), r.end(), out_all + o);
    }
    return PFB_OK;
}

extern "C" int pfb_mr_ctx_from_residue(pfb_mr_ctx_t *c, const uint64_t *d_x, uint64_t *out_all) {
    if (!out_all) {
        pfb::set_error("pfb_mr_ctx_from_residue: bad argument");
        return PFB_E_ARG;
    }
    const int rc = ctx_launch(c, d_x, nullptr, c ? c->d_tmp : nullptr, c ? c->n16 : 0, CTX_FROM, nullptr);
    if (rc) return rc;
    PFB_CUDA(cudaMemcpy(out_all, c->d_tmp, (size_t)c->n * c->n16 * 8, cudaMemcpyDeviceToHost));
    return PFB_OK;
}

extern "C" int pfb_mr_ctx_check_passed(pfb_mr_ctx_t *c, const uint64_t *d_r, uint8_t *d_passed, void *stream) {
    if (!c || !d_r || !d_passed) {
        pfb::set_error("pfb_mr_ctx_check_passed: bad argument");
        return PFB_E_ARG;
    }
    PFB_CUDA(cudaSetDevice(c->e->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : cudaStreamLegacy;
    ctx_check_kernel<<<c->n, 256, 0, st>>>(d_r, c->d_one, c->d_nm1, d_passed, c->n16);
    PFB_CUDA(cudaGetLastError());
    return PFB_OK;
}

extern "C" int pfb_mr_ctx_modsq(pfb_mr_ctx_t *c, const uint64_t *d_a, uint64_t *d_out, void *stream) {
    return ctx_launch(c, d_a, nullptr, d_out, c ? c->n16 : 0, CTX_MODSQ, stream);
}

extern "C" int pfb_mr_ctx_modmul(pfb_mr_ctx_t *c, const uint64_t *d_a, const uint64_t *d_b, uint64_t *d_out,
                                 void *stream) {
    return ctx_launch(c, d_a, d_b, d_out, c ? c->n16 : 0, CTX_MODMUL, stream);
}

extern "C" int pfb_mr_ctx_sq_raw(pfb_mr_ctx_t *c, const uint64_t *d_a, uint64_t *d_out, void *stream) {
    return ctx_launch(c, d_a, nullptr, d_out, c ? 2 * c->n16 + 16 : 0, CTX_RAW_SQ, stream);
}

extern "C" int pfb_mr_ctx_mul_raw(pfb_mr_ctx_t *c, const uint64_t *d_a, const uint64_t *d_b, uint64_t *d_out,
                                  void *stream) {
    return ctx_launch(c, d_a, d_b, d_out, c ? 2 * c->n16 + 16 : 0, CTX_RAW_MUL, stream);
}

// ---------------------------------------------------------------------------
// Measurement: two forms of one radix-16 pass (radix_probe.cuh).

extern "C" int pfb_mr_radix16_forms(pfb_mr_t *e, int ctas, int reps, double *ms_butterfly, double *ms_tensor,
                                    long long *mismatches, int *tensor_error) {
    if (!e || ctas <= 0 || reps <= 0 || !ms_butterfly || !ms_tensor || !mismatches || !tensor_error) {
        pfb::set_error("pfb_mr_radix16_forms: bad argument");
        return PFB_E_ARG;
    }
    PFB_CUDA(cudaSetDevice(e->device));
    const uint32_t P[2] = {P1, P2};
    // host tables: the operand image of the byte planes of F, omega_n^t, floor(2^64 / p)
    std::vector<uint8_t> fa(RP_OPND, 0);
    std::vector<uint32_t> wn(4 * (size_t)RP_N);
    RpTables t{};
    for (int pr = 0; pr < 2; pr++) {
        const uint64_t p = P[pr];
        uint64_t om = 1, b = 3, ex = (p - 1) >> LOG_LMAX;  // order 2^15
        for (; ex; ex >>= 1, b = b * b % p)
            if (ex & 1) om = om * b % p;
        const uint64_t wn1 = om * om % p;  // order 2^14
        uint64_t w16 = 1;
        for (int i = 0; i < RP_N / 16; i++) w16 = w16 * wn1 % p;  // order 16
        uint32_t *wv = wn.data() + (size_t)(2 * pr) * RP_N, *ws = wv + RP_N;
        uint64_t a = 1;
        for (int i = 0; i < RP_N; i++, a = a * wn1 % p) {
            wv[i] = (uint32_t)a;
            ws[i] = (uint32_t)(((uint64_t)a << 32) / p);
        }
        for (int k = 0; k < 16; k++) {
            uint64_t wk = 1;
            for (int i = 0; i < k; i++) wk = wk * w16 % p;
            uint64_t f = 1;
            for (int m = 0; m < 16; m++, f = f * wk % p)
                for (int byte = 0; byte < 4; byte++) fa[rp_off(pr * 64 + k * 4 + byte, m)] = (uint8_t)(f >> (8 * byte));
        }
        t.mu[pr] = ~0ull / p;
    }
    const size_t nx = (size_t)ctas * RP_N;
    uint32_t *d_x = nullptr, *d_yb = nullptr, *d_yt = nullptr, *d_wn = nullptr;
    uint8_t *d_fa = nullptr;
    int *d_err = nullptr;
    cudaError_t ce = cudaMalloc(&d_x, nx * 4);
    if (ce == cudaSuccess) ce = cudaMalloc(&d_yb, 2 * nx * 4);
    if (ce == cudaSuccess) ce = cudaMalloc(&d_yt, 2 * nx * 4);
    if (ce == cudaSuccess) ce = cudaMalloc(&d_wn, wn.size() * 4);
    if (ce == cudaSuccess) ce = cudaMalloc(&d_fa, fa.size());
    if (ce == cudaSuccess) ce = cudaMalloc(&d_err, sizeof(int));
    auto release = [&]() {
        cudaFree(d_x);
        cudaFree(d_yb);
        cudaFree(d_yt);
        cudaFree(d_wn);
        cudaFree(d_fa);
        cudaFree(d_err);
    };
    if (ce != cudaSuccess) {
        release();
        return pfb::cuda_fail(ce, "pfb_mr_radix16_forms: allocation", __FILE__, __LINE__);
    }
    std::vector<uint32_t> hx(nx);
    uint64_t st = 0x9E3779B97F4A7C15ull;
    for (auto &v : hx) {
        st = st * 6364136223846793005ull + 1442695040888963407ull;
        v = (uint32_t)(st >> 40) & LIMB_MASK;
    }
    float ms_b = 0.f, ms_t = 0.f;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    do {
        if ((ce = cudaMemcpy(d_x, hx.data(), nx * 4, cudaMemcpyHostToDevice)) != cudaSuccess) break;
        if ((ce = cudaMemcpy(d_wn, wn.data(), wn.size() * 4, cudaMemcpyHostToDevice)) != cudaSuccess) break;
        if ((ce = cudaMemcpy(d_fa, fa.data(), fa.size(), cudaMemcpyHostToDevice)) != cudaSuccess) break;
        if ((ce = cudaMemset(d_err, 0, sizeof(int))) != cudaSuccess) break;
        t.fa = d_fa;
        for (int pr = 0; pr < 2; pr++) {
            t.wn[pr] = d_wn + (size_t)(2 * pr) * RP_N;
            t.wnsh[pr] = t.wn[pr] + RP_N;
        }
        const int smem_b = (int)(2 * (RP_N + RP_N / 32) * sizeof(uint32_t));
        if ((ce = cudaFuncSetAttribute(rp_butterfly_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_b)) !=
            cudaSuccess)
            break;
        if ((ce = cudaFuncSetAttribute(rp_tensor_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, RP_SMEM)) !=
            cudaSuccess)
            break;
        if ((ce = cudaEventCreate(&e0)) != cudaSuccess || (ce = cudaEventCreate(&e1)) != cudaSuccess) break;
        cudaStream_t s = e->stream;
        for (int form = 0; form < 2 && ce == cudaSuccess; form++) {
            for (int r = -1; r < reps; r++) {  // one untimed launch first
                if (r == 0) cudaEventRecord(e0, s);
                if (form == 0) rp_butterfly_kernel<<<ctas, THREADS, smem_b, s>>>(d_x, d_yb, e->tw);
                else rp_tensor_kernel<<<ctas, THREADS, RP_SMEM, s>>>(d_x, d_yt, t, d_err);
            }
            cudaEventRecord(e1, s);
            if ((ce = cudaEventSynchronize(e1)) != cudaSuccess) break;
            if ((ce = cudaGetLastError()) != cudaSuccess) break;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            (form == 0 ? ms_b : ms_t) = ms / reps;
        }
        if (ce != cudaSuccess) break;
        std::vector<uint32_t> yb(2 * nx), yt(2 * nx);
        if ((ce = cudaMemcpy(yb.data(), d_yb, yb.size() * 4, cudaMemcpyDeviceToHost)) != cudaSuccess) break;
        if ((ce = cudaMemcpy(yt.data(), d_yt, yt.size() * 4, cudaMemcpyDeviceToHost)) != cudaSuccess) break;
        if ((ce = cudaMemcpy(tensor_error, d_err, sizeof(int), cudaMemcpyDeviceToHost)) != cudaSuccess) break;
        long long bad = 0;
        for (size_t i = 0; i < yb.size(); i++) bad += yb[i] != yt[i];
        *mismatches = bad;
    } while (0);
    int rc = PFB_OK;
    if (ce != cudaSuccess) rc = pfb::cuda_fail(ce, "pfb_mr_radix16_forms", __FILE__, __LINE__);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    release();
    *ms_butterfly = ms_b;
    *ms_tensor = ms_t;
    return rc;
}
