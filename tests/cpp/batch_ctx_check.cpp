// The reference's BatchModCtx correctness checks (miller_rabin_gpu/
// correctness_tests.cuh:96-639), restated against include/batch_mod_ctx.cuh
// and checked with GMP: for "small" (x = i + 2), "large" (x = N - i - 2) and
// "rand" (xorshift limbs, reduced mod N) operands -- the reference's three
// value sets, seeds 0xDEADBEEF12345678 / 0xCAFEBABE87654321 (:138-179):
//   roundtrip       from_residue(to_residue(x)) == x
//   raw_sq/raw_mul  sq_no_redc / mul_no_redc of the working forms == mpz_mul
//   modsq/modmul    == x^2 mod N, x y mod N
//   chain16         16 squarings == x^65536 mod N
//   powm            x^0xDEADBEEF by square-and-multiply == mpz_powm_ui (:578-639)
//   nm1_sq          (N - 1)^2 == 1
//   check_passed    1 and N - 1 pass, a random residue does not
// Moduli: n_batch = 4 random odd numbers per size, built through the mpz_t
// constructor.  Prints "name size pass fail" per check.
#include <cstdio>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>  // cudaMalloc(T **), as the reference's .cu callers see it
#include <gmp.h>

#include "batch_mod_ctx.cuh"

static uint64_t xs(uint64_t &s) {
    s ^= s << 13;
    s ^= s >> 7;
    s ^= s << 17;
    return s;
}

static void to_mpz(mpz_t out, const uint64_t *l, int n) {
    std::vector<uint16_t> w(n);
    for (int i = 0; i < n; i++) w[i] = (uint16_t)l[i];
    mpz_import(out, n, -1, 2, 0, 0, w.data());
}

static void from_mpz(uint64_t *out, int n, const mpz_t x) {
    std::vector<uint16_t> w((mpz_sizeinbase(x, 2) + 15) / 16 + 2, 0);
    size_t cnt = 0;
    mpz_export(w.data(), &cnt, -1, 2, 0, 0, x);
    for (int i = 0; i < n; i++) out[i] = i < (int)cnt ? w[i] : 0;
}

static bool eq(const uint64_t *a, const uint64_t *b, int n) { return memcmp(a, b, sizeof(uint64_t) * n) == 0; }

#define CU(x)                                                              \
    do {                                                                   \
        if ((x) != cudaSuccess) {                                          \
            fprintf(stderr, "CUDA error %s at %d\n", #x, __LINE__);         \
            return 2;                                                      \
        }                                                                  \
    } while (0)

int main(int argc, char **argv) {
    std::vector<int> sizes = {512, 2048, 20000, 166000, 332000};
    if (argc > 1) {
        sizes.clear();
        for (int i = 1; i < argc; i++) sizes.push_back(atoi(argv[i]));
    }
    uint64_t seed = 0xDEADBEEF12345678ull;
    for (int bits : sizes) {
        const int nb = 4;
        std::vector<__mpz_struct> store(nb);
        std::vector<mpz_t *> nums(nb);
        for (int i = 0; i < nb; i++) {
            mpz_t *p = reinterpret_cast<mpz_t *>(&store[i]);
            mpz_init(*p);
            std::vector<uint16_t> w((bits + 15) / 16);
            for (auto &x : w) x = (uint16_t)xs(seed);
            const int top = (bits - 1) % 16;
            w.back() = (uint16_t)((w.back() & ((1u << top) - 1u)) | (1u << top));
            w[0] |= 1u;
            mpz_import(*p, w.size(), -1, 2, 0, 0, w.data());
            nums[i] = p;
        }
        BatchModCtx mont(nums, 0);
        const int n = mont.n_limbs, ns = mont.n_sum;
        const size_t tb = (size_t)nb * n * sizeof(Data64);
        std::vector<uint64_t> N_h((size_t)nb * n);
        CU(cudaMemcpy(N_h.data(), mont.d_N, tb, cudaMemcpyDeviceToHost));
        // the three value sets (correctness_tests.cuh:110-179)
        std::vector<uint64_t> xsm((size_t)nb * n, 0), xlg((size_t)nb * n), xrn((size_t)nb * n);
        uint64_t s2 = 0xCAFEBABE87654321ull;
        mpz_t Nm, t, u, v;
        mpz_init(Nm);
        mpz_init(t);
        mpz_init(u);
        mpz_init(v);
        for (int i = 0; i < nb; i++) {
            xsm[(size_t)i * n] = (uint64_t)(i + 2);
            to_mpz(Nm, N_h.data() + (size_t)i * n, n);
            mpz_sub_ui(t, Nm, (unsigned long)(i + 2));
            from_mpz(xlg.data() + (size_t)i * n, n, t);
            std::vector<uint64_t> r(n);
            for (auto &x : r) x = xs(s2) & 0xFFFFu;
            to_mpz(t, r.data(), n);
            mpz_mod(t, t, Nm);
            from_mpz(xrn.data() + (size_t)i * n, n, t);
        }
        Data64 *d_x, *d_y, *d_o, *d_w;
        uint8_t *d_p;
        CU(cudaMalloc(&d_x, tb));
        CU(cudaMalloc(&d_y, tb));
        CU(cudaMalloc(&d_o, (size_t)nb * ns * sizeof(Data64)));
        CU(cudaMalloc(&d_w, tb));
        CU(cudaMalloc(&d_p, nb));
        struct Set {
            const std::vector<uint64_t> *x, *y;
            const char *name;
        } sets[] = {{&xsm, &xrn, "small"}, {&xlg, &xsm, "large"}, {&xrn, &xlg, "rand"}};
        for (const Set &st : sets) {
            std::vector<uint64_t> xm, ym, got, raw((size_t)nb * ns);
            mont.to_residue_batch(*st.x, xm);
            mont.to_residue_batch(*st.y, ym);
            int pass[8] = {0}, fail[8] = {0};
            const char *names[8] = {"roundtrip", "raw_sq", "raw_mul", "modsq", "modmul", "chain16", "powm", "nm1_sq"};
            auto tally = [&](int k, bool ok) { (ok ? pass : fail)[k]++; };
            CU(cudaMemcpy(d_x, xm.data(), tb, cudaMemcpyHostToDevice));
            CU(cudaMemcpy(d_y, ym.data(), tb, cudaMemcpyHostToDevice));
            mont.from_residue_batch(d_x, got);
            for (int i = 0; i < nb; i++) tally(0, eq(got.data() + (size_t)i * n, st.x->data() + (size_t)i * n, n));
            // raw products of the working forms (correctness_tests.cuh:252-312)
            mont.sq_no_redc_batch(d_x, d_o);
            CU(cudaMemcpy(raw.data(), d_o, raw.size() * 8, cudaMemcpyDeviceToHost));
            for (int i = 0; i < nb; i++) {
                std::vector<uint64_t> ref(ns);
                to_mpz(t, xm.data() + (size_t)i * n, n);
                mpz_mul(u, t, t);
                from_mpz(ref.data(), ns, u);
                tally(1, eq(raw.data() + (size_t)i * ns, ref.data(), ns));
            }
            mont.mul_no_redc_batch(d_x, d_y, d_o);
            CU(cudaMemcpy(raw.data(), d_o, raw.size() * 8, cudaMemcpyDeviceToHost));
            for (int i = 0; i < nb; i++) {
                std::vector<uint64_t> ref(ns);
                to_mpz(t, xm.data() + (size_t)i * n, n);
                to_mpz(v, ym.data() + (size_t)i * n, n);
                mpz_mul(u, t, v);
                from_mpz(ref.data(), ns, u);
                tally(2, eq(raw.data() + (size_t)i * ns, ref.data(), ns));
            }
            // modsq / modmul (:314-357)
            mont.modsq_batch(d_x, d_w);
            mont.from_residue_batch(d_w, got);
            for (int i = 0; i < nb; i++) {
                std::vector<uint64_t> ref(n);
                to_mpz(Nm, N_h.data() + (size_t)i * n, n);
                to_mpz(t, st.x->data() + (size_t)i * n, n);
                mpz_mul(u, t, t);
                mpz_mod(u, u, Nm);
                from_mpz(ref.data(), n, u);
                tally(3, eq(got.data() + (size_t)i * n, ref.data(), n));
            }
            mont.modmul_batch(d_x, d_y, d_w);
            mont.from_residue_batch(d_w, got);
            for (int i = 0; i < nb; i++) {
                std::vector<uint64_t> ref(n);
                to_mpz(Nm, N_h.data() + (size_t)i * n, n);
                to_mpz(t, st.x->data() + (size_t)i * n, n);
                to_mpz(v, st.y->data() + (size_t)i * n, n);
                mpz_mul(u, t, v);
                mpz_mod(u, u, Nm);
                from_mpz(ref.data(), n, u);
                tally(4, eq(got.data() + (size_t)i * n, ref.data(), n));
            }
            // 16 chained squarings (:359-396)
            CU(cudaMemcpy(d_w, d_x, tb, cudaMemcpyDeviceToDevice));
            for (int k = 0; k < 16; k++) {
                mont.modsq_batch(d_w, d_o);
                CU(cudaMemcpy(d_w, d_o, tb, cudaMemcpyDeviceToDevice));
            }
            mont.from_residue_batch(d_w, got);
            for (int i = 0; i < nb; i++) {
                std::vector<uint64_t> ref(n);
                to_mpz(Nm, N_h.data() + (size_t)i * n, n);
                to_mpz(t, st.x->data() + (size_t)i * n, n);
                mpz_powm_ui(u, t, 65536ul, Nm);
                from_mpz(ref.data(), n, u);
                tally(5, eq(got.data() + (size_t)i * n, ref.data(), n));
            }
            // x^0xDEADBEEF, left to right (:578-639)
            const unsigned long E = 0xDEADBEEFul;
            CU(cudaMemcpy(d_w, d_x, tb, cudaMemcpyDeviceToDevice));
            for (int bit = 30; bit >= 0; bit--) {
                mont.modsq_batch(d_w, d_o);
                if ((E >> bit) & 1ul) mont.modmul_batch(d_o, d_x, d_w);
                else CU(cudaMemcpy(d_w, d_o, tb, cudaMemcpyDeviceToDevice));
            }
            mont.from_residue_batch(d_w, got);
            for (int i = 0; i < nb; i++) {
                std::vector<uint64_t> ref(n);
                to_mpz(Nm, N_h.data() + (size_t)i * n, n);
                to_mpz(t, st.x->data() + (size_t)i * n, n);
                mpz_powm_ui(u, t, E, Nm);
                from_mpz(ref.data(), n, u);
                tally(6, eq(got.data() + (size_t)i * n, ref.data(), n));
            }
            // (N - 1)^2 == 1 in the working form, and check_passed
            mont.modsq_batch(mont.d_Nm1_res, d_w);
            std::vector<uint64_t> one((size_t)nb * n), w2((size_t)nb * n);
            CU(cudaMemcpy(one.data(), mont.d_one_res, tb, cudaMemcpyDeviceToHost));
            CU(cudaMemcpy(w2.data(), d_w, tb, cudaMemcpyDeviceToHost));
            for (int i = 0; i < nb; i++) tally(7, eq(w2.data() + (size_t)i * n, one.data() + (size_t)i * n, n));
            for (int k = 0; k < 8; k++) printf("%s %d %s %d %d\n", names[k], bits, st.name, pass[k], fail[k]);
            uint8_t pz[4];
            int cp = 0, cf = 0;
            for (const Data64 *src : {mont.d_one_res, mont.d_Nm1_res, (const Data64 *)d_y}) {
                mont.check_passed(src, d_p);
                CU(cudaMemcpy(pz, d_p, nb, cudaMemcpyDeviceToHost));
                const bool want = src != d_y;
                for (int i = 0; i < nb; i++) {
                    // a "rand"/"small"/"large" residue may equal 1 or N - 1 only by construction: x = 1 never
                    // occurs (x >= 2), x = N - 1 never (x <= N - 2)
                    (pz[i] == (uint8_t)want ? cp : cf)++;
                }
            }
            printf("check_passed %d %s %d %d\n", bits, st.name, cp, cf);
        }
        cudaFree(d_x);
        cudaFree(d_y);
        cudaFree(d_o);
        cudaFree(d_w);
        cudaFree(d_p);
        mpz_clear(Nm);
        mpz_clear(t);
        mpz_clear(u);
        mpz_clear(v);
        for (int i = 0; i < nb; i++) mpz_clear(*nums[i]);
    }
    return 0;
}
