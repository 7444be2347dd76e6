/*
 * Stand-in <gmp.h> for building the reference's CPU transforms in an image
 * that ships libgmp.so.10 but not its development header.  Test
 * infrastructure only (used by oracle/Makefile for oracle/_ref).
 *
 * Declares the documented public GMP 6 ABI for the handful of mpz entry
 * points the reference headers, oracle/ref_harness.cpp and
 * oracle/genefer_harness.cpp call.  Each
 * mpz_* name maps to the __gmpz_* symbol exported by libgmp.so.10.
 */
#pragma once

#include <stddef.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef unsigned long int mp_limb_t;
typedef long int mp_size_t;
typedef unsigned long int mp_bitcnt_t;

typedef struct
{
	int _mp_alloc;
	int _mp_size;
	mp_limb_t *_mp_d;
} __mpz_struct;

typedef __mpz_struct mpz_t[1];
typedef __mpz_struct *mpz_ptr;
typedef const __mpz_struct *mpz_srcptr;

#define mpz_init __gmpz_init
#define mpz_init_set __gmpz_init_set
#define mpz_init_set_ui __gmpz_init_set_ui
#define mpz_clear __gmpz_clear
#define mpz_set_ui __gmpz_set_ui
#define mpz_mul_2exp __gmpz_mul_2exp
#define mpz_sqrt __gmpz_sqrt
#define mpz_div_2exp __gmpz_fdiv_q_2exp
#define mpz_fdiv_q_2exp __gmpz_fdiv_q_2exp
#define mpz_mod_2exp __gmpz_fdiv_r_2exp
#define mpz_fdiv_r_2exp __gmpz_fdiv_r_2exp
#define mpz_get_d __gmpz_get_d
#define mpz_fdiv_ui __gmpz_fdiv_ui
#define mpz_inp_raw __gmpz_inp_raw
#define mpz_out_raw __gmpz_out_raw
#define mpz_ui_pow_ui __gmpz_ui_pow_ui
#define mpz_sizeinbase __gmpz_sizeinbase
#define mpz_tstbit __gmpz_tstbit
#define mpz_add __gmpz_add
#define mpz_export __gmpz_export
#define mpz_add_ui __gmpz_add_ui
#define mpz_addmul __gmpz_addmul
#define mpz_cmp __gmpz_cmp
#define mpz_mul __gmpz_mul
#define mpz_mul_ui __gmpz_mul_ui
#define mpz_sub __gmpz_sub

void __gmpz_init(mpz_ptr);
void __gmpz_init_set(mpz_ptr, mpz_srcptr);
void __gmpz_init_set_ui(mpz_ptr, unsigned long int);
void __gmpz_clear(mpz_ptr);
void __gmpz_set_ui(mpz_ptr, unsigned long int);
void __gmpz_mul_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
void __gmpz_sqrt(mpz_ptr, mpz_srcptr);
void __gmpz_fdiv_q_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
void __gmpz_fdiv_r_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
double __gmpz_get_d(mpz_srcptr);
unsigned long int __gmpz_fdiv_ui(mpz_srcptr, unsigned long int);
size_t __gmpz_inp_raw(mpz_ptr, FILE *);
size_t __gmpz_out_raw(FILE *, mpz_srcptr);
void __gmpz_ui_pow_ui(mpz_ptr, unsigned long int, unsigned long int);
size_t __gmpz_sizeinbase(mpz_srcptr, int);
int __gmpz_tstbit(mpz_srcptr, mp_bitcnt_t);
void __gmpz_add(mpz_ptr, mpz_srcptr, mpz_srcptr);
void *__gmpz_export(void *, size_t *, int, size_t, int, size_t, mpz_srcptr);
void __gmpz_add_ui(mpz_ptr, mpz_srcptr, unsigned long int);
void __gmpz_addmul(mpz_ptr, mpz_srcptr, mpz_srcptr);
int __gmpz_cmp(mpz_srcptr, mpz_srcptr);
void __gmpz_mul(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_mul_ui(mpz_ptr, mpz_srcptr, unsigned long int);
void __gmpz_sub(mpz_ptr, mpz_srcptr, mpz_srcptr);

#define mpz_sgn(z) ((z)->_mp_size < 0 ? -1 : (z)->_mp_size > 0)

#ifdef __cplusplus
}
#endif
