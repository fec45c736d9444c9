/* TEST INFRASTRUCTURE ONLY.  This image has MPFR 4 and GMP 6 runtime libraries (libmpfr.so.6, libgmp.so.10) but no
 * headers, so the bridge test compiles against these declarations, written from the public MPFR 4 and GMP 6 manuals:
 * the mpfr_t / mpz_t layouts are part of their stable ABIs, and every name below is an exported function of the
 * libraries (the real headers define some of them as macros too).  A user's build uses the real <mpfr.h>. */
#ifndef LIMBFORGE_TEST_MPFR_DECL_H
#define LIMBFORGE_TEST_MPFR_DECL_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
#define GMP_NUMB_BITS 64
#define GMP_NAIL_BITS 0
typedef unsigned long mp_limb_t;
typedef struct { int _mp_alloc; int _mp_size; mp_limb_t* _mp_d; } __mpz_struct;
typedef __mpz_struct mpz_t[1];
typedef __mpz_struct* mpz_ptr;
typedef const __mpz_struct* mpz_srcptr;
void __gmpz_init(mpz_ptr);
void __gmpz_clear(mpz_ptr);
void __gmpz_import(mpz_ptr, size_t, int, size_t, int, size_t, const void*);
void* __gmpz_export(void*, size_t*, int, size_t, int, size_t, mpz_srcptr);
size_t __gmpz_sizeinbase(mpz_srcptr, int);
void __gmpz_neg(mpz_ptr, mpz_srcptr);
void __gmpz_mul_2exp(mpz_ptr, mpz_srcptr, unsigned long);
#define mpz_init __gmpz_init
#define mpz_clear __gmpz_clear
#define mpz_import __gmpz_import
#define mpz_export __gmpz_export
#define mpz_sizeinbase __gmpz_sizeinbase
#define mpz_neg __gmpz_neg
#define mpz_mul_2exp __gmpz_mul_2exp

typedef long mpfr_prec_t;
typedef int mpfr_sign_t;
typedef long mpfr_exp_t;
typedef struct { mpfr_prec_t _mpfr_prec; mpfr_sign_t _mpfr_sign; mpfr_exp_t _mpfr_exp; mp_limb_t* _mpfr_d; } __mpfr_struct;
typedef __mpfr_struct mpfr_t[1];
typedef __mpfr_struct* mpfr_ptr;
typedef const __mpfr_struct* mpfr_srcptr;
typedef enum { MPFR_RNDN = 0, MPFR_RNDZ, MPFR_RNDU, MPFR_RNDD, MPFR_RNDA } mpfr_rnd_t;
typedef enum { MPFR_NAN_KIND = 0, MPFR_INF_KIND = 1, MPFR_ZERO_KIND = 2, MPFR_REGULAR_KIND = 3 } mpfr_kind_t;
typedef enum { MPFR_FREE_LOCAL_CACHE = 1, MPFR_FREE_GLOBAL_CACHE = 2 } mpfr_free_cache_t;

void mpfr_init2(mpfr_ptr, mpfr_prec_t);
void mpfr_clear(mpfr_ptr);
mpfr_prec_t mpfr_get_prec(mpfr_srcptr);
mpfr_exp_t mpfr_get_exp(mpfr_srcptr);
int mpfr_set_exp(mpfr_ptr, mpfr_exp_t);
int mpfr_number_p(mpfr_srcptr);
int mpfr_regular_p(mpfr_srcptr);
int mpfr_zero_p(mpfr_srcptr);
int mpfr_nan_p(mpfr_srcptr);
int mpfr_inf_p(mpfr_srcptr);
int mpfr_signbit(mpfr_srcptr);
int mpfr_sgn(mpfr_srcptr);
void mpfr_set_nan(mpfr_ptr);
void mpfr_set_inf(mpfr_ptr, int);
void mpfr_set_zero(mpfr_ptr, int);
int mpfr_set(mpfr_ptr, mpfr_srcptr, mpfr_rnd_t);
int mpfr_set_si(mpfr_ptr, long, mpfr_rnd_t);
int mpfr_set_z_2exp(mpfr_ptr, mpz_srcptr, mpfr_exp_t, mpfr_rnd_t);
mpfr_exp_t mpfr_get_z_2exp(mpz_ptr, mpfr_srcptr);
int mpfr_set_str(mpfr_ptr, const char*, int, mpfr_rnd_t);
int mpfr_equal_p(mpfr_srcptr, mpfr_srcptr);
int mpfr_cmp(mpfr_srcptr, mpfr_srcptr);
int mpfr_sub(mpfr_ptr, mpfr_srcptr, mpfr_srcptr, mpfr_rnd_t);
int mpfr_ui_div(mpfr_ptr, unsigned long, mpfr_srcptr, mpfr_rnd_t);
int mpfr_mul_2si(mpfr_ptr, mpfr_srcptr, long, mpfr_rnd_t);
void* mpfr_custom_get_significand(mpfr_srcptr);
void mpfr_custom_init_set(mpfr_ptr, int, mpfr_exp_t, mpfr_prec_t, void*);
void mpfr_custom_init(void*, mpfr_prec_t);
size_t mpfr_custom_get_size(mpfr_prec_t);
void mpfr_set_inexflag(void);
void mpfr_clear_inexflag(void);
int mpfr_inexflag_p(void);
mpfr_exp_t mpfr_get_emin(void);
mpfr_exp_t mpfr_get_emax(void);
int mpfr_set_emin(mpfr_exp_t);
int mpfr_set_emax(mpfr_exp_t);
mpfr_exp_t mpfr_get_emin_min(void);
mpfr_exp_t mpfr_get_emax_max(void);
void mpfr_free_cache2(mpfr_free_cache_t);
#ifdef __cplusplus
}
#endif
/* The real header also defines the field accessors as macros over the documented layout (zero, NaN and infinity
 * encoded in the exponent field as its minimum + 1, + 2, + 3), so a build against it inlines them; so does this one. */
#define LIMBFORGE_TEST_MPFR_EXP_ZERO (-0x7fffffffffffffffL - 1L + 1)
#define LIMBFORGE_TEST_MPFR_EXP_INF (-0x7fffffffffffffffL - 1L + 3)
#define mpfr_get_prec(x) ((mpfr_prec_t)(x)->_mpfr_prec)
#define mpfr_get_exp(x) ((mpfr_exp_t)(x)->_mpfr_exp)
#define mpfr_signbit(x) ((x)->_mpfr_sign < 0)
#define mpfr_zero_p(x) ((x)->_mpfr_exp == LIMBFORGE_TEST_MPFR_EXP_ZERO)
#define mpfr_regular_p(x) ((x)->_mpfr_exp > LIMBFORGE_TEST_MPFR_EXP_INF)
#define mpfr_number_p(x) ((x)->_mpfr_exp > LIMBFORGE_TEST_MPFR_EXP_INF || (x)->_mpfr_exp == LIMBFORGE_TEST_MPFR_EXP_ZERO)
#define mpfr_custom_get_significand(x) ((void*)(x)->_mpfr_d)
#endif
