/*
 * gmp.h (declaration shim) -- the documented GMP mpz interface that the reference's
 * CPU sources call, declared for linking against the system libgmp.so.10 (GMP 6.x ABI),
 * whose development header is not installed in this image.  Used only to build the
 * reference CPU path as the test oracle (oracle/ref/build_ref.py); never part of the
 * product.
 */
#ifndef CUFE_ORACLE_GMP_SHIM_H
#define CUFE_ORACLE_GMP_SHIM_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef unsigned long int mp_limb_t;
typedef unsigned long int mp_bitcnt_t;
typedef struct {
  int _mp_alloc;
  int _mp_size;
  mp_limb_t *_mp_d;
} __mpz_struct;
typedef __mpz_struct mpz_t[1];
typedef __mpz_struct *mpz_ptr;
typedef const __mpz_struct *mpz_srcptr;

void __gmpz_init(mpz_ptr);
void __gmpz_clear(mpz_ptr);
void __gmpz_set(mpz_ptr, mpz_srcptr);
void __gmpz_set_ui(mpz_ptr, unsigned long int);
int __gmpz_set_str(mpz_ptr, const char *, int);
void __gmpz_add(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_add_ui(mpz_ptr, mpz_srcptr, unsigned long int);
void __gmpz_sub(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_mul(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_mul_ui(mpz_ptr, mpz_srcptr, unsigned long int);
void __gmpz_mul_2exp(mpz_ptr, mpz_srcptr, mp_bitcnt_t);
void __gmpz_mod(mpz_ptr, mpz_srcptr, mpz_srcptr);
unsigned long int __gmpz_fdiv_r_ui(mpz_ptr, mpz_srcptr, unsigned long int);
unsigned long int __gmpz_fdiv_ui(mpz_srcptr, unsigned long int);
unsigned long int __gmpz_fdiv_q_ui(mpz_ptr, mpz_srcptr, unsigned long int);
unsigned long int __gmpz_fdiv_qr_ui(mpz_ptr, mpz_ptr, mpz_srcptr, unsigned long int);
void __gmpz_fdiv_qr(mpz_ptr, mpz_ptr, mpz_srcptr, mpz_srcptr);
int __gmpz_cmp(mpz_srcptr, mpz_srcptr);
int __gmpz_cmp_ui(mpz_srcptr, unsigned long int);
double __gmpz_get_d(mpz_srcptr);
unsigned long int __gmpz_get_ui(mpz_srcptr);
char *__gmpz_get_str(char *, int, mpz_srcptr);
size_t __gmpz_sizeinbase(mpz_srcptr, int);
int __gmp_printf(const char *, ...);

#define mpz_init __gmpz_init
#define mpz_clear __gmpz_clear
#define mpz_set __gmpz_set
#define mpz_set_ui __gmpz_set_ui
#define mpz_set_str __gmpz_set_str
#define mpz_add __gmpz_add
#define mpz_add_ui __gmpz_add_ui
#define mpz_sub __gmpz_sub
#define mpz_mul __gmpz_mul
#define mpz_mul_ui __gmpz_mul_ui
#define mpz_mul_2exp __gmpz_mul_2exp
#define mpz_mod __gmpz_mod
#define mpz_mod_ui __gmpz_fdiv_r_ui
#define mpz_fdiv_ui __gmpz_fdiv_ui
#define mpz_fdiv_q_ui __gmpz_fdiv_q_ui
#define mpz_fdiv_qr_ui __gmpz_fdiv_qr_ui
#define mpz_fdiv_qr __gmpz_fdiv_qr
#define mpz_cmp __gmpz_cmp
#define mpz_cmp_ui __gmpz_cmp_ui
#define mpz_get_d __gmpz_get_d
#define mpz_get_ui __gmpz_get_ui
#define mpz_get_str __gmpz_get_str
#define mpz_sizeinbase __gmpz_sizeinbase
#define gmp_printf __gmp_printf
#ifdef __cplusplus
}
#endif
#endif
