/*
 * Declarations-only header for the subset of GMP's documented public API
 * that the reference CPU kernel (pfvs/fp_kernel/fp_kernel.h and
 * pfvs/fp_kernel/pfv_lattice.h) calls.  The image ships the GMP runtime
 * (libgmp.so.10) but not its development header; this file lets the
 * reference sources compile unmodified against that runtime, for the
 * oracle's reference build only (oracle/_ref).  Nothing in the product
 * includes it.
 *
 * Types follow GMP's documented ABI on LP64 Linux: an integer is
 * {alloc, size, limb pointer}; a rational is {numerator, denominator}.
 * Every function is the library's exported __gmpz_* / __gmpq_* symbol,
 * bound to the documented mpz_* / mpq_* name by a macro.  mpz_sgn is a
 * macro in GMP's documented interface and is one here too.
 */
#ifndef PFVS_ORACLE_GMP_DECLS_H
#define PFVS_ORACLE_GMP_DECLS_H

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

typedef struct {
    __mpz_struct _mp_num;
    __mpz_struct _mp_den;
} __mpq_struct;
typedef __mpq_struct mpq_t[1];
typedef __mpq_struct *mpq_ptr;
typedef const __mpq_struct *mpq_srcptr;

/* integers */
void   __gmpz_init(mpz_ptr);
void   __gmpz_init_set(mpz_ptr, mpz_srcptr);
void   __gmpz_init_set_si(mpz_ptr, long);
void   __gmpz_init_set_ui(mpz_ptr, unsigned long);
void   __gmpz_clear(mpz_ptr);
void   __gmpz_set(mpz_ptr, mpz_srcptr);
void   __gmpz_set_si(mpz_ptr, long);
void   __gmpz_set_ui(mpz_ptr, unsigned long);
void   __gmpz_swap(mpz_ptr, mpz_ptr);
void   __gmpz_neg(mpz_ptr, mpz_srcptr);
void   __gmpz_add(mpz_ptr, mpz_srcptr, mpz_srcptr);
void   __gmpz_mul(mpz_ptr, mpz_srcptr, mpz_srcptr);
void   __gmpz_mul_si(mpz_ptr, mpz_srcptr, long);
void   __gmpz_addmul_ui(mpz_ptr, mpz_srcptr, unsigned long);
void   __gmpz_submul_ui(mpz_ptr, mpz_srcptr, unsigned long);
void   __gmpz_submul(mpz_ptr, mpz_srcptr, mpz_srcptr);
void   __gmpz_divexact(mpz_ptr, mpz_srcptr, mpz_srcptr);
void   __gmpz_fdiv_q(mpz_ptr, mpz_srcptr, mpz_srcptr);
void   __gmpz_gcd(mpz_ptr, mpz_srcptr, mpz_srcptr);
int    __gmpz_cmpabs(mpz_srcptr, mpz_srcptr);
int    __gmpz_fits_slong_p(mpz_srcptr);
long   __gmpz_get_si(mpz_srcptr);
size_t __gmpz_sizeinbase(mpz_srcptr, int);
void   __gmpz_import(mpz_ptr, size_t, int, size_t, int, size_t, const void *);
void  *__gmpz_export(void *, size_t *, int, size_t, int, size_t, mpz_srcptr);

#define mpz_init          __gmpz_init
#define mpz_init_set      __gmpz_init_set
#define mpz_init_set_si   __gmpz_init_set_si
#define mpz_init_set_ui   __gmpz_init_set_ui
#define mpz_clear         __gmpz_clear
#define mpz_set           __gmpz_set
#define mpz_set_si        __gmpz_set_si
#define mpz_set_ui        __gmpz_set_ui
#define mpz_swap          __gmpz_swap
#define mpz_neg           __gmpz_neg
#define mpz_add           __gmpz_add
#define mpz_mul           __gmpz_mul
#define mpz_mul_si        __gmpz_mul_si
#define mpz_addmul_ui     __gmpz_addmul_ui
#define mpz_submul_ui     __gmpz_submul_ui
#define mpz_submul        __gmpz_submul
#define mpz_divexact      __gmpz_divexact
#define mpz_fdiv_q        __gmpz_fdiv_q
#define mpz_gcd           __gmpz_gcd
#define mpz_cmpabs        __gmpz_cmpabs
#define mpz_fits_slong_p  __gmpz_fits_slong_p
#define mpz_get_si        __gmpz_get_si
#define mpz_sizeinbase    __gmpz_sizeinbase
#define mpz_import        __gmpz_import
#define mpz_export        __gmpz_export
#define mpz_sgn(z)        ((z)->_mp_size < 0 ? -1 : (z)->_mp_size > 0)

/* rationals */
void   __gmpq_init(mpq_ptr);
void   __gmpq_inits(mpq_ptr, ...);
void   __gmpq_clear(mpq_ptr);
void   __gmpq_clears(mpq_ptr, ...);
void   __gmpq_set_num(mpq_ptr, mpz_srcptr);
void   __gmpq_set_den(mpq_ptr, mpz_srcptr);
void   __gmpq_set_si(mpq_ptr, long, unsigned long);
void   __gmpq_canonicalize(mpq_ptr);
double __gmpq_get_d(mpq_srcptr);
void   __gmpq_add(mpq_ptr, mpq_srcptr, mpq_srcptr);
void   __gmpq_sub(mpq_ptr, mpq_srcptr, mpq_srcptr);
void   __gmpq_mul(mpq_ptr, mpq_srcptr, mpq_srcptr);

#define mpq_init          __gmpq_init
#define mpq_inits         __gmpq_inits
#define mpq_clear         __gmpq_clear
#define mpq_clears        __gmpq_clears
#define mpq_set_num       __gmpq_set_num
#define mpq_set_den       __gmpq_set_den
#define mpq_set_si        __gmpq_set_si
#define mpq_canonicalize  __gmpq_canonicalize
#define mpq_get_d         __gmpq_get_d
#define mpq_add           __gmpq_add
#define mpq_sub           __gmpq_sub
#define mpq_mul           __gmpq_mul

#ifdef __cplusplus
}
#endif

#endif
