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
#include "mr_device.cuh"
#include "pfb_mr.h"

namespace pfb {
namespace mr {

__constant__ CrtConsts c_crt;

// State of one candidate in device memory.
struct JobDev {
    uint32_t *x;          // H limbs: Montgomery residue (working value)
    uint32_t *res;        // H limbs: canonical residue a^E mod N (output)
    uint32_t *nph;        // [2][L] NTT_L(N')
    uint32_t *nh;         // [2][H] NTT_H(N)
    const uint32_t *npl;  // H limbs of N' (set-up input)
    const uint32_t *nl;   // H limbs of N
    const uint32_t *exp;  // exponent, 32-bit words, little-endian
    int logl;
    int cursor;   // next exponent bit (MSB first); phase 0 while >= 0
    int extra;    // squarings left in phase 2 (s - 1 for a strong test)
    int phase;    // 0 exponent loop, 1 first check, 2 squarings r < s, 3 done
    uint32_t base;
    int mode;     // 0 modular power only, 1 strong test
    int verdict;  // 1 probable prime, 0 composite
    int steps;    // steps taken (diagnostics)
};

__host__ __device__ inline size_t smem_words(int logl) {
    const size_t L = (size_t)1 << logl, H = L / 2;
    return 2 * (L + L / 32) + 2 * H;
}
inline size_t smem_bytes(int logl) {
    return smem_words(logl) * sizeof(uint32_t) + sizeof(CarrySmem) + 16;
}

__device__ __forceinline__ void carve(uint32_t *raw, int logl, Smem &sm, uint32_t *&Y) {
    const int L = 1 << logl, H = L >> 1;
    sm.A0 = raw;
    sm.A1 = raw + L + L / 32;
    sm.X = sm.A1 + L + L / 32;
    Y = sm.X + H;
    uintptr_t c = (uintptr_t)(Y + H);
    c = (c + 15) & ~(uintptr_t)15;
    sm.cs = (CarrySmem *)c;
}

__global__ void __launch_bounds__(THREADS, 1) prep_kernel(JobDev *jobs, Twiddles tw) {
    extern __shared__ __align__(16) uint32_t raw[];
    const JobDev jb = jobs[blockIdx.x];
    if (jb.phase == 3) return;
    Smem sm;
    uint32_t *Y;
    carve(raw, jb.logl, sm, Y);
    const int L = 1 << jb.logl, H = L >> 1;
    for (int i = threadIdx.x; i < L; i += blockDim.x) {
        const uint32_t v = i < H ? jb.npl[i] : 0u;
        sm.A0[pad(i)] = v;
        sm.A1[pad(i)] = v;
    }
    __syncthreads();
    dif(sm.A0, sm.A1, jb.logl, tw);
    for (int i = threadIdx.x; i < L; i += blockDim.x) {
        jb.nph[i] = red2(sm.A0[pad(i)], P1);
        jb.nph[L + i] = red2(sm.A1[pad(i)], P2);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < H; i += blockDim.x) {
        sm.A0[pad(i)] = jb.nl[i];
        sm.A1[pad(i)] = jb.nl[i];
    }
    __syncthreads();
    dif(sm.A0, sm.A1, jb.logl - 1, tw);
    for (int i = threadIdx.x; i < H; i += blockDim.x) {
        jb.nh[i] = red2(sm.A0[pad(i)], P1);
        jb.nh[H + i] = red2(sm.A1[pad(i)], P2);
    }
}

// Canonical residue of X (Montgomery form) into Y: Y = X R^-1 mod N.
__device__ void canonical(const Smem &sm, uint32_t *Y, const Cand &cd, const uint32_t *nl, const Twiddles &tw) {
    const int H = 1 << (cd.logl - 1);
    for (int i = threadIdx.x; i < H; i += blockDim.x) Y[i] = sm.X[i];
    __syncthreads();
    Smem s2 = sm;
    s2.X = Y;
    mont_step(s2, cd, false, 1u, tw, c_crt);
    // REDC(X) lies in [0, N]; it is N only when X == 0 (mod N), e.g. a base
    // that is a multiple of N.  Map it to 0.
    bool eqn = true;
    for (int i = threadIdx.x; i < H; i += blockDim.x) eqn = eqn && (Y[i] == nl[i]);
    if (__syncthreads_and(eqn))
        for (int i = threadIdx.x; i < H; i += blockDim.x) Y[i] = 0u;
    __syncthreads();
}

__global__ void __launch_bounds__(THREADS, 1) step_kernel(JobDev *jobs, int max_steps, Twiddles tw) {
    extern __shared__ __align__(16) uint32_t raw[];
    JobDev *jp = jobs + blockIdx.x;
    const JobDev jb = *jp;
    if (jb.phase == 3) return;
    Smem sm;
    uint32_t *Y;
    carve(raw, jb.logl, sm, Y);
    const int H = 1 << (jb.logl - 1);
    const Cand cd{jb.nph, jb.nh, jb.logl};
    for (int i = threadIdx.x; i < H; i += blockDim.x) sm.X[i] = jb.x[i];
    __syncthreads();

    int cursor = jb.cursor, phase = jb.phase, extra = jb.extra, verdict = jb.verdict, steps = 0;
    while (steps < max_steps && phase != 3) {
        if (phase == 0) {
            const uint32_t bit = (__ldg(jb.exp + (cursor >> 5)) >> (cursor & 31)) & 1u;
            mont_step(sm, cd, true, bit ? jb.base : 1u, tw, c_crt);
            cursor--;
            if (cursor < 0) phase = 1;
        } else {
            if (phase == 2) {
                mont_step(sm, cd, true, 1u, tw, c_crt);
                extra--;
            }
            canonical(sm, Y, cd, jb.nl, tw);
            // compare with 1 and N - 1 (N odd: N - 1 differs from N in limb 0 only)
            bool one = true, nm1 = true;
            for (int i = threadIdx.x; i < H; i += blockDim.x) {
                const uint32_t y = Y[i], nli = jb.nl[i];
                one = one && (y == (i == 0 ? 1u : 0u));
                nm1 = nm1 && (y == (i == 0 ? nli - 1u : nli));
            }
            const int all_one = __syncthreads_and(one);
            const int all_nm1 = __syncthreads_and(nm1);
            if (phase == 1)
                for (int i = threadIdx.x; i < H; i += blockDim.x) jb.res[i] = Y[i];
            if (jb.mode == 0) {
                phase = 3;
            } else if (all_nm1 || (phase == 1 && all_one)) {
                verdict = 1;
                phase = 3;
            } else if (extra <= 0) {
                verdict = 0;
                phase = 3;
            } else {
                phase = 2;
            }
        }
        steps++;
    }
    for (int i = threadIdx.x; i < H; i += blockDim.x) jb.x[i] = sm.X[i];
    if (threadIdx.x == 0) {
        jp->cursor = cursor;
        jp->phase = phase;
        jp->extra = extra;
        jp->verdict = verdict;
        jp->steps = jb.steps + steps;
    }
}

// ---------------------------------------------------------------- host ----

static uint32_t powmod_h(uint64_t b, uint64_t e, uint32_t p) {
    uint64_t r = 1;
    b %= p;
    while (e) {
        if (e & 1) r = r * b % p;
        b = b * b % p;
        e >>= 1;
    }
    return (uint32_t)r;
}
static uint32_t shoup_c(uint32_t w, uint32_t p) { return (uint32_t)(((uint64_t)w << 32) / p); }

struct HostPrep {
    int ok = 0;  // 1 = valid
    int logl = 0;
    int s = 0;
    std::vector<uint32_t> x0, npl, nl, exp;
    int cursor = 0;
    int n16 = 0;  // limbs of N (16-bit)
};

static int choose_logl(size_t nbits, uint32_t base) {
    const int abits = 32 - __builtin_clz(base);
    for (int lg = LOG_LMIN; lg <= LOG_LCTA; lg++) {
        const size_t rbits = (size_t)LIMB_BITS << (lg - 1);
        if (rbits >= nbits + 2 + 2 * (size_t)abits) return lg;
    }
    return -1;
}

// mode 1: exponent d of N - 1 = 2^s d; mode 0: exponent given.
static void host_prep(const pfb_mr_number_t &num, uint32_t base, int mode, const pfb_mr_number_t *ex,
                      HostPrep &hp) {
    using namespace pfb::big;
    hp.ok = 0;
    if (!num.limbs || num.n_limbs <= 0) return;
    Words N = from_u16(num.limbs, (size_t)num.n_limbs);
    const size_t nb = bit_length(N);
    if (nb < 2 || !(N[0] & 1ull) || nb > (size_t)PFB_MR_MAX_BITS) return;
    const int lg = choose_logl(nb, base);
    if (lg < 0) return;
    const size_t H = (size_t)1 << (lg - 1);
    const size_t rbits = LIMB_BITS * H;
    Words E;
    int s = 0;
    if (mode == 1) {
        Words nm1 = sub_small(N, 1);
        while (!test_bit(nm1, (size_t)s)) s++;
        E = shr(nm1, (size_t)s);
    } else {
        if (!ex || !ex->limbs || ex->n_limbs <= 0) return;
        E = from_u16(ex->limbs, (size_t)ex->n_limbs);
        if (E.empty()) return;
    }
    hp.logl = lg;
    hp.s = s;
    hp.n16 = num.n_limbs;
    hp.npl.assign(H, 0);
    hp.nl.assign(H, 0);
    hp.x0.assign(H, 0);
    to_limbs(neg_inv_pow2(N, rbits), LIMB_BITS, hp.npl.data(), H);
    to_limbs(N, LIMB_BITS, hp.nl.data(), H);
    to_limbs(pow2_mod(rbits, N), LIMB_BITS, hp.x0.data(), H);
    const size_t eb = bit_length(E);
    hp.cursor = (int)eb - 1;
    hp.exp.assign((eb + 31) / 32 + 1, 0);
    for (size_t i = 0; i < eb; i++)
        if (test_bit(E, i)) hp.exp[i / 32] |= 1u << (i % 32);
    hp.ok = 1;
}

}  // namespace mr
}  // namespace pfb

using namespace pfb::mr;

struct pfb_mr {
    int device = 0;
    int num_sms = 0;
    cudaStream_t stream = nullptr;
    uint32_t *d_tw = nullptr;
    Twiddles tw{};
    uint8_t *d_arena = nullptr;
    size_t arena_bytes = 0;
};

static int build_tables(pfb_mr *e) {
    const int half = 1 << (LOG_LMAX - 1);
    std::vector<uint32_t> h((size_t)8 * half);
    const uint32_t P[2] = {P1, P2};
    for (int pr = 0; pr < 2; pr++) {
        const uint32_t p = P[pr];
        const uint32_t om = powmod_h(3, (p - 1) >> LOG_LMAX, p);
        const uint32_t omi = powmod_h(om, p - 2, p);
        uint32_t *w = h.data() + (size_t)(4 * pr + 0) * half, *wsh = w + half, *wi = wsh + half, *wish = wi + half;
        uint64_t a = 1, b = 1;
        for (int k = 0; k < half; k++) {
            w[k] = (uint32_t)a;
            wsh[k] = shoup_c((uint32_t)a, p);
            wi[k] = (uint32_t)b;
            wish[k] = shoup_c((uint32_t)b, p);
            a = a * om % p;
            b = b * omi % p;
        }
    }
    PFB_CUDA(cudaMalloc(&e->d_tw, h.size() * sizeof(uint32_t)));
    PFB_CUDA(cudaMemcpy(e->d_tw, h.data(), h.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
    for (int pr = 0; pr < 2; pr++) {
        uint32_t *base = e->d_tw + (size_t)(4 * pr) * half;
        e->tw.w[pr] = base;
        e->tw.wsh[pr] = base + half;
        e->tw.wi[pr] = base + 2 * half;
        e->tw.wish[pr] = base + 3 * half;
    }
    CrtConsts cc{};
    const uint32_t ip1 = powmod_h(P1 % P2, P2 - 2, P2);
    const uint32_t two32_1 = (uint32_t)((1ull << 32) % P1), two32_2 = (uint32_t)((1ull << 32) % P2);
    for (int lg = 0; lg <= LOG_LMAX; lg++) {
        const uint32_t s1 = (uint32_t)((uint64_t)two32_1 * powmod_h(1ull << lg, P1 - 2, P1) % P1);
        const uint32_t s2 = (uint32_t)((uint64_t)two32_2 * powmod_h(1ull << lg, P2 - 2, P2) % P2);
        cc.s1[lg] = s1;
        cc.s1sh[lg] = shoup_c(s1, P1);
        cc.k2[lg] = (uint32_t)((uint64_t)s2 * ip1 % P2);
        cc.k2sh[lg] = shoup_c(cc.k2[lg], P2);
    }
    cc.k1 = ip1;
    cc.k1sh = shoup_c(ip1, P2);
    for (int pr = 0; pr < 2; pr++) {
        uint32_t inv = 1;  // p^-1 mod 2^32 by Newton
        for (int i = 0; i < 5; i++) inv *= 2u - P[pr] * inv;
        cc.pinv[pr] = 0u - inv;
    }
    PFB_CUDA(cudaMemcpyToSymbol(c_crt, &cc, sizeof(cc)));
    return PFB_OK;
}

extern "C" int pfb_mr_create(pfb_mr_t **out, int device) {
    if (!out) {
        pfb::set_error("pfb_mr_create: null out");
        return PFB_E_ARG;
    }
    *out = nullptr;
    pfb_mr *e = new pfb_mr();
    e->device = device;
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
        const int mx = (int)smem_bytes(LOG_LCTA);
        ce = cudaFuncSetAttribute(step_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
        if (ce == cudaSuccess) ce = cudaFuncSetAttribute(prep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
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
    cudaFree(e->d_arena);
    delete e;
}

namespace {

// Per-candidate device layout inside the arena (32-bit words).
struct Layout {
    size_t x, res, nph, nh, npl, nl, exp, total;
};

Layout layout_for(const HostPrep &hp) {
    const size_t L = (size_t)1 << hp.logl, H = L / 2;
    Layout l{};
    size_t o = 0;
    auto take = [&](size_t words) {
        const size_t at = o;
        o += (words + 63) & ~(size_t)63;  // 256-byte alignment
        return at;
    };
    l.x = take(H);
    l.res = take(H);
    l.nph = take(2 * L);
    l.nh = take(2 * H);
    l.npl = take(H);
    l.nl = take(H);
    l.exp = take(hp.exp.size());
    l.total = o;
    return l;
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

int run_jobs(pfb_mr *e, const pfb_mr_number_t *nums, int n, uint32_t base, int mode,
             const pfb_mr_number_t *exps, int8_t *verdict, uint16_t *residue, int residue_stride) {
    if (!e || !nums || n <= 0 || base < 2 || base > 0xFFFFu) {
        pfb::set_error("pfb_mr: bad argument (n=%d base=%u)", n, base);
        return PFB_E_ARG;
    }
    if (residue && residue_stride <= 0) {
        pfb::set_error("pfb_mr: residue_stride must be > 0");
        return PFB_E_ARG;
    }
    PFB_CUDA(cudaSetDevice(e->device));
    std::vector<HostPrep> hp;
    prep_all(nums, n, base, mode, exps, hp);
    std::vector<Layout> lay(n);
    size_t total = 0;
    int maxlog = LOG_LMIN, n_ok = 0;
    long long max_steps = 0;
    for (int i = 0; i < n; i++) {
        if (verdict) verdict[i] = -1;
        if (!hp[i].ok) continue;
        lay[i] = layout_for(hp[i]);
        total += lay[i].total;
        maxlog = std::max(maxlog, hp[i].logl);
        max_steps = std::max(max_steps, (long long)hp[i].cursor + 2 + hp[i].s);
        n_ok++;
    }
    const size_t job_bytes = ((size_t)n * sizeof(JobDev) + 255) & ~(size_t)255;
    const size_t need = job_bytes + total * sizeof(uint32_t);
    if (need > e->arena_bytes) {
        cudaFree(e->d_arena);
        e->d_arena = nullptr;
        e->arena_bytes = 0;
        cudaError_t ce = cudaMalloc(&e->d_arena, need);
        if (ce != cudaSuccess) {
            pfb::set_error("pfb_mr: cannot allocate %zu bytes", need);
            return PFB_E_NOMEM;
        }
        e->arena_bytes = need;
    }
    JobDev *d_jobs = (JobDev *)e->d_arena;
    uint32_t *d_words = (uint32_t *)(e->d_arena + job_bytes);
    std::vector<JobDev> jobs(n);
    size_t off = 0;
    for (int i = 0; i < n; i++) {
        JobDev &j = jobs[i];
        memset(&j, 0, sizeof(j));
        if (!hp[i].ok) {
            j.phase = 3;
            continue;
        }
        uint32_t *b = d_words + off;
        const Layout &l = lay[i];
        j.x = b + l.x;
        j.res = b + l.res;
        j.nph = b + l.nph;
        j.nh = b + l.nh;
        j.npl = b + l.npl;
        j.nl = b + l.nl;
        j.exp = b + l.exp;
        j.logl = hp[i].logl;
        j.cursor = hp[i].cursor;
        j.extra = mode == 1 ? hp[i].s - 1 : 0;
        j.phase = 0;
        j.base = base;
        j.mode = mode;
        const size_t H = hp[i].x0.size();
        PFB_CUDA(cudaMemcpyAsync(j.x, hp[i].x0.data(), H * 4, cudaMemcpyHostToDevice, e->stream));
        PFB_CUDA(cudaMemcpyAsync((void *)j.npl, hp[i].npl.data(), H * 4, cudaMemcpyHostToDevice, e->stream));
        PFB_CUDA(cudaMemcpyAsync((void *)j.nl, hp[i].nl.data(), H * 4, cudaMemcpyHostToDevice, e->stream));
        PFB_CUDA(cudaMemcpyAsync((void *)j.exp, hp[i].exp.data(), hp[i].exp.size() * 4, cudaMemcpyHostToDevice,
                                 e->stream));
        off += l.total;
    }
    PFB_CUDA(cudaMemcpyAsync(d_jobs, jobs.data(), n * sizeof(JobDev), cudaMemcpyHostToDevice, e->stream));
    if (n_ok) {
        const size_t sm = smem_bytes(maxlog);
        prep_kernel<<<n, THREADS, sm, e->stream>>>(d_jobs, e->tw);
        PFB_CUDA(cudaGetLastError());
        const int chunk = 2048;
        for (long long done = 0; done < max_steps; done += chunk) {
            step_kernel<<<n, THREADS, sm, e->stream>>>(d_jobs, chunk, e->tw);
            PFB_CUDA(cudaGetLastError());
        }
    }
    PFB_CUDA(cudaMemcpyAsync(jobs.data(), d_jobs, n * sizeof(JobDev), cudaMemcpyDeviceToHost, e->stream));
    PFB_CUDA(cudaStreamSynchronize(e->stream));
    std::vector<uint32_t> r22;
    for (int i = 0; i < n; i++) {
        if (!hp[i].ok) continue;
        if (jobs[i].phase != 3) {
            pfb::set_error("pfb_mr: candidate %d did not finish", i);
            return PFB_E_STATE;
        }
        if (verdict) verdict[i] = (int8_t)(mode == 1 ? jobs[i].verdict : 0);
        if (residue) {
            const size_t H = hp[i].x0.size();
            r22.resize(H);
            PFB_CUDA(cudaMemcpy(r22.data(), jobs[i].res, H * 4, cudaMemcpyDeviceToHost));
            pfb::big::Words r = pfb::big::from_limbs(r22.data(), LIMB_BITS, H);
            pfb::big::to_u16(r, residue + (size_t)i * residue_stride, (size_t)residue_stride);
        }
    }
    return PFB_OK;
}

}  // namespace

extern "C" int pfb_mr_test(pfb_mr_t *e, const pfb_mr_number_t *nums, int n, uint32_t base, int8_t *verdict,
                           uint16_t *residue, int residue_stride) {
    return run_jobs(e, nums, n, base, 1, nullptr, verdict, residue, residue_stride);
}

extern "C" int pfb_mr_powm(pfb_mr_t *e, const pfb_mr_number_t *nums, int n, uint32_t base,
                           const pfb_mr_number_t *exps, uint16_t *residue, int residue_stride) {
    if (!exps || !residue) {
        pfb::set_error("pfb_mr_powm: exps and residue are required");
        return PFB_E_ARG;
    }
    return run_jobs(e, nums, n, base, 0, exps, nullptr, residue, residue_stride);
}

extern "C" long long pfb_mr_test_cost(const uint16_t *limbs, int n_limbs) {
    if (!limbs || n_limbs <= 0) return -1;
    pfb::big::Words N = pfb::big::from_u16(limbs, (size_t)n_limbs);
    const size_t nb = pfb::big::bit_length(N);
    if (nb < 2) return -1;
    return (long long)nb;  // ~ bits(d) squarings + one conversion
}
