/*
 * Declaration-only stand-in for <gmp.h> (TEST INFRASTRUCTURE, oracle side).
 *
 * The image ships the GMP 6.3 runtime (libgmp.so.10) but no development
 * header.  This file declares the handful of documented public mpz_* entry
 * points that the oracle and the reference's miller_rabin.c call, with the
 * signatures from the GMP manual ("Integer Functions").  GMP exports them
 * under the __gmpz_ prefix, so each public name is mapped to its symbol.
 * Nothing here is product code: only oracle/ and tests link against it.
 */
#ifndef PFB_ORACLE_GMP_DECL_H
#define PFB_ORACLE_GMP_DECL_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef unsigned long mp_limb_t;
typedef long mp_size_t;
typedef unsigned long mp_bitcnt_t;

typedef struct {
    int _mp_alloc;
    int _mp_size;
    mp_limb_t *_mp_d;
} __mpz_struct;

typedef __mpz_struct mpz_t[1];
typedef __mpz_struct *mpz_ptr;
typedef const __mpz_struct *mpz_srcptr;

#define mpz_init            __gmpz_init
#define mpz_inits           __gmpz_inits
#define mpz_init_set        __gmpz_init_set
#define mpz_clear           __gmpz_clear
#define mpz_clears          __gmpz_clears
#define mpz_set             __gmpz_set
#define mpz_set_ui          __gmpz_set_ui
#define mpz_get_ui          __gmpz_get_ui
#define mpz_ui_pow_ui       __gmpz_ui_pow_ui
#define mpz_mul             __gmpz_mul
#define mpz_mul_ui          __gmpz_mul_ui
#define mpz_mul_2exp        __gmpz_mul_2exp
#define mpz_add             __gmpz_add
#define mpz_add_ui          __gmpz_add_ui
#define mpz_sub             __gmpz_sub
#define mpz_sub_ui          __gmpz_sub_ui
#define mpz_mod             __gmpz_mod
#define mpz_tdiv_q_2exp     __gmpz_tdiv_q_2exp
#define mpz_tdiv_r_2exp     __gmpz_tdiv_r_2exp
#define mpz_powm            __gmpz_powm
#define mpz_powm_ui         __gmpz_powm_ui
#define mpz_cmp             __gmpz_cmp
#define mpz_cmp_ui          __gmpz_cmp_ui
#define mpz_sizeinbase      __gmpz_sizeinbase
#define mpz_scan1           __gmpz_scan1
#define mpz_tstbit          __gmpz_tstbit
#define mpz_probab_prime_p  __gmpz_probab_prime_p
#define mpz_nextprime       __gmpz_nextprime
#define mpz_import          __gmpz_import
#define mpz_export          __gmpz_export
#define mpz_invert          __gmpz_invert

void mpz_init(mpz_ptr);
void mpz_inits(mpz_ptr, ...);
void mpz_init_set(mpz_ptr, mpz_srcptr);
void mpz_clear(mpz_ptr);
void mpz_clears(mpz_ptr, ...);
void mpz_set(mpz_ptr, mpz_srcptr);
void mpz_set_ui(mpz_ptr, unsigned long);
unsigned long mpz_get_ui(mpz_srcptr);
void mpz_ui_pow_ui(mpz_ptr, unsigned long, unsigned long);
void mpz_mul(mpz_ptr, mpz_srcptr, mpz_srcptr);
void mpz_mul_ui(mpz_ptr, mpz_srcptr, unsigned long);
void mpz_mul_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
void mpz_add(mpz_ptr, mpz_srcptr, mpz_srcptr);
void mpz_add_ui(mpz_ptr, mpz_srcptr, unsigned long);
void mpz_sub(mpz_ptr, mpz_srcptr, mpz_srcptr);
void mpz_sub_ui(mpz_ptr, mpz_srcptr, unsigned long);
void mpz_mod(mpz_ptr, mpz_srcptr, mpz_srcptr);
void mpz_tdiv_q_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
void mpz_tdiv_r_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
void mpz_powm(mpz_ptr, mpz_srcptr, mpz_srcptr, mpz_srcptr);
void mpz_powm_ui(mpz_ptr, mpz_srcptr, unsigned long, mpz_srcptr);
int mpz_cmp(mpz_srcptr, mpz_srcptr);
int mpz_cmp_ui(mpz_srcptr, unsigned long);
size_t mpz_sizeinbase(mpz_srcptr, int);
mp_bitcnt_t mpz_scan1(mpz_srcptr, mp_bitcnt_t);
int mpz_tstbit(mpz_srcptr, mp_bitcnt_t);
int mpz_probab_prime_p(mpz_srcptr, int);
void mpz_nextprime(mpz_ptr, mpz_srcptr);
void mpz_import(mpz_ptr, size_t, int, size_t, int, size_t, const void *);
void *mpz_export(void *, size_t *, int, size_t, int, size_t, mpz_srcptr);
int mpz_invert(mpz_ptr, mpz_srcptr, mpz_srcptr);

#define mpz_even_p(z) (((z)->_mp_size == 0) || !((z)->_mp_d[0] & 1))
#define mpz_odd_p(z)  (!mpz_even_p(z))

#ifdef __cplusplus
}
#endif
#endif
