/*
 * Independent MPFR oracle (TEST INFRASTRUCTURE ONLY).  The reference's tests replay every
 * operation in MPFR (tests/reference.hpp:33-116): real ops with mpfr_add/sub/mul/sqr/sqrt/div
 * RNDN, fused ops with mpfr_fma/mpfr_fms, dot2_add and exact dots as exact 2*bits products
 * summed by one mpfr_sum.  This file does the same through the installed runtime libraries
 * (libmpfr.so.6, libgmp.so.10); this image has no MPFR/GMP headers, so the few declarations
 * needed are written here from the public MPFR 4 / GMP 6 manuals (mpfr_t and mpz_t layouts
 * are part of their stable ABI).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef long mpfr_prec_t; typedef int mpfr_sign_t; typedef long mpfr_exp_t; typedef unsigned long mp_limb_t;
typedef struct { mpfr_prec_t prec; mpfr_sign_t sign; mpfr_exp_t exp; mp_limb_t* d; } mpfr_struct;
typedef mpfr_struct* mpfr_ptr;
typedef struct { int alloc; int size; mp_limb_t* d; } mpz_struct;
typedef mpz_struct* mpz_ptr;
enum { RNDN = 0 };

extern void mpfr_init2(mpfr_ptr, mpfr_prec_t);
extern void mpfr_clear(mpfr_ptr);
extern int mpfr_set_z_2exp(mpfr_ptr, mpz_ptr, mpfr_exp_t, int);
extern mpfr_exp_t mpfr_get_z_2exp(mpz_ptr, mpfr_ptr);
extern int mpfr_add(mpfr_ptr, mpfr_ptr, mpfr_ptr, int);
extern int mpfr_sub(mpfr_ptr, mpfr_ptr, mpfr_ptr, int);
extern int mpfr_mul(mpfr_ptr, mpfr_ptr, mpfr_ptr, int);
extern int mpfr_div(mpfr_ptr, mpfr_ptr, mpfr_ptr, int);
extern int mpfr_sqr(mpfr_ptr, mpfr_ptr, int);
extern int mpfr_sqrt(mpfr_ptr, mpfr_ptr, int);
extern int mpfr_fma(mpfr_ptr, mpfr_ptr, mpfr_ptr, mpfr_ptr, int);
extern int mpfr_fms(mpfr_ptr, mpfr_ptr, mpfr_ptr, mpfr_ptr, int);
extern int mpfr_neg(mpfr_ptr, mpfr_ptr, int);
extern int mpfr_set(mpfr_ptr, mpfr_ptr, int);
extern int mpfr_sum(mpfr_ptr, mpfr_ptr*, unsigned long, int);
extern void mpfr_set_zero(mpfr_ptr, int);
extern int mpfr_set_emin(mpfr_exp_t);
extern int mpfr_set_emax(mpfr_exp_t);
extern void __gmpz_init(mpz_ptr);
extern void __gmpz_clear(mpz_ptr);
extern void __gmpz_import(mpz_ptr, size_t, int, size_t, int, size_t, const void*);
extern void* __gmpz_export(void*, size_t*, int, size_t, int, size_t, mpz_ptr);
extern size_t __gmpz_sizeinbase(mpz_ptr, int);
extern void __gmpz_neg(mpz_ptr, mpz_ptr);

typedef uint32_t word;
#define EMAX 1000000000L

static void zero_num(word* o, int n, word st) { memset(o, 0, sizeof(word) * (size_t)(n + 3)); o[n + 2] = st; }

static void widen_range(void) { mpfr_set_emin(-3000000000L); mpfr_set_emax(3000000000L); }

/* x must have status 0 */
static void to_mp(mpfr_ptr out, const word* x, int n) {
    int sign = (int32_t)x[n + 1];
    if (!sign) { mpfr_set_zero(out, 1); return; }
    mpz_struct z; __gmpz_init(&z);
    __gmpz_import(&z, (size_t)n, -1, 4, 0, 0, x);
    if (sign < 0) __gmpz_neg(&z, &z);
    mpfr_set_z_2exp(out, &z, (mpfr_exp_t)(int32_t)x[n] - (32L * n - 1), RNDN);
    __gmpz_clear(&z);
}
/* Number from an MPFR value already rounded to 32n bits; |exponent| > 1e9 -> exponent_overflow */
static void from_mp(word* o, mpfr_ptr x, int n) {
    mpz_struct z; __gmpz_init(&z);
    mpfr_exp_t e = mpfr_get_z_2exp(&z, x);
    if (z.size == 0) { zero_num(o, n, 0); __gmpz_clear(&z); return; }
    int sign = z.size < 0 ? -1 : 1;
    if (sign < 0) __gmpz_neg(&z, &z);
    long bits = (long)__gmpz_sizeinbase(&z, 2);
    long ex = e + bits - 1;                                   /* value in [2^ex, 2^(ex+1)) */
    if (ex > EMAX || ex < -EMAX) { zero_num(o, n, 2); __gmpz_clear(&z); return; }
    word buf[40]; memset(buf, 0, sizeof buf); size_t cnt = 0;
    __gmpz_export(buf, &cnt, -1, 4, 0, 0, &z);
    /* left-align the significand in n words */
    long shift = 32L * n - bits;
    zero_num(o, n, 0);
    for (int i = 0; i < n; ++i) {
        long src = 32L * i - shift; word v = 0;
        if (src >= 0) { long w = src / 32; int s = (int)(src % 32); if (w < 40) v = buf[w] >> s; if (s && w + 1 < 40) v |= buf[w + 1] << (32 - s); }
        else if (src > -32) v = buf[0] << (-src);
        o[i] = v;
    }
    o[n] = (word)(int32_t)ex; o[n + 1] = (word)sign;
    __gmpz_clear(&z);
}

/* op codes as limbforge::Operation for the real ops: 0 add 1 sub 2 mul 3 div 7 square 8 sqrt */
int mpo_real(int bits, int op, const word* a, const word* b, word* out, size_t count) {
    const int n = bits / 32; const size_t E = (size_t)n + 3; widen_range();
    mpfr_struct x, y, r; mpfr_init2(&x, bits); mpfr_init2(&y, bits); mpfr_init2(&r, bits);
    for (size_t i = 0; i < count; ++i) {
        const word* p = a + i * E; const word* q = b ? b + i * E : NULL; word* o = out + i * E;
        int unary = op == 7 || op == 8;
        word st = p[n + 2] | (unary ? 0 : q[n + 2]);
        if (st) { zero_num(o, n, st); continue; }
        if (op == 3 && !(int32_t)q[n + 1]) { zero_num(o, n, 1); continue; }
        if (op == 8 && (int32_t)p[n + 1] < 0) { zero_num(o, n, 4); continue; }
        to_mp(&x, p, n); if (!unary) to_mp(&y, q, n);
        switch (op) {
        case 0: mpfr_add(&r, &x, &y, RNDN); break;
        case 1: mpfr_sub(&r, &x, &y, RNDN); break;
        case 2: mpfr_mul(&r, &x, &y, RNDN); break;
        case 3: mpfr_div(&r, &x, &y, RNDN); break;
        case 7: mpfr_sqr(&r, &x, RNDN); break;
        case 8: mpfr_sqrt(&r, &x, RNDN); break;
        default: return 1;
        }
        from_mp(o, &r, n);
    }
    mpfr_clear(&x); mpfr_clear(&y); mpfr_clear(&r);
    return 0;
}
int mpo_fused(int bits, int subtract, const word* a, const word* b, const word* c, word* out, size_t count) {
    const int n = bits / 32; const size_t E = (size_t)n + 3; widen_range();
    mpfr_struct x, y, z, r; mpfr_init2(&x, bits); mpfr_init2(&y, bits); mpfr_init2(&z, bits); mpfr_init2(&r, bits);
    for (size_t i = 0; i < count; ++i) {
        const word* p = a + i * E; const word* q = b + i * E; const word* s = c + i * E; word* o = out + i * E;
        word st = p[n + 2] | q[n + 2] | s[n + 2];
        if (st) { zero_num(o, n, st); continue; }
        to_mp(&x, p, n); to_mp(&y, q, n); to_mp(&z, s, n);
        if (subtract) mpfr_fms(&r, &x, &y, &z, RNDN); else mpfr_fma(&r, &x, &y, &z, RNDN);
        from_mp(o, &r, n);
    }
    mpfr_clear(&x); mpfr_clear(&y); mpfr_clear(&z); mpfr_clear(&r);
    return 0;
}
/* RN(c -/+ sum a_k b_k) or RN(sum) (c NULL): exact 2*bits products, one mpfr_sum
 * (tests/reference.hpp:74-94).  Strides in elements. */
int mpo_dot(int bits, const word* c, int subtract, const word* a, long sa, const word* b, long sb, size_t K, word* out) {
    const int n = bits / 32; const long E = n + 3; widen_range();
    word st = c ? c[n + 2] : 0;
    for (size_t k = 0; k < K; ++k) st |= a[(long)k * sa * E + n + 2] | b[(long)k * sb * E + n + 2];
    if (st) { zero_num(out, n, st); return 0; }
    mpfr_struct* p = (mpfr_struct*)malloc(sizeof(mpfr_struct) * (K + 1));
    mpfr_ptr* terms = (mpfr_ptr*)malloc(sizeof(mpfr_ptr) * (K + 1));
    mpfr_struct x, y, r; mpfr_init2(&x, bits); mpfr_init2(&y, bits); mpfr_init2(&r, bits);
    for (size_t k = 0; k < K; ++k) {
        mpfr_init2(&p[k], 2L * bits); terms[k] = &p[k];
        to_mp(&x, a + (long)k * sa * E, n); to_mp(&y, b + (long)k * sb * E, n);
        mpfr_mul(&p[k], &x, &y, RNDN);
        if (subtract) mpfr_neg(&p[k], &p[k], RNDN);
    }
    size_t T = K;
    if (c) { mpfr_init2(&p[K], 2L * bits); terms[K] = &p[K]; to_mp(&p[K], c, n); T = K + 1; }
    mpfr_sum(&r, terms, T, RNDN);
    from_mp(out, &r, n);
    for (size_t k = 0; k < T; ++k) mpfr_clear(&p[k]);
    mpfr_clear(&x); mpfr_clear(&y); mpfr_clear(&r); free(p); free(terms);
    return 0;
}
/* RN(a*b + c*d + e) (tests/reference.hpp:64-72) */
int mpo_dot2_add(int bits, const word* a, const word* b, const word* c, const word* d, const word* e, word* out, size_t count) {
    const int n = bits / 32; const size_t E = (size_t)n + 3; widen_range();
    mpfr_struct xa, xb, xc, xd, xe, p, q, r; mpfr_ptr t[3];
    mpfr_init2(&xa, bits); mpfr_init2(&xb, bits); mpfr_init2(&xc, bits); mpfr_init2(&xd, bits); mpfr_init2(&xe, bits);
    mpfr_init2(&p, 2L * bits); mpfr_init2(&q, 2L * bits); mpfr_init2(&r, bits);
    for (size_t i = 0; i < count; ++i) {
        const word *A = a + i * E, *B = b + i * E, *C = c + i * E, *D = d + i * E, *F = e + i * E; word* o = out + i * E;
        word st = A[n + 2] | B[n + 2] | C[n + 2] | D[n + 2] | F[n + 2];
        if (st) { zero_num(o, n, st); continue; }
        to_mp(&xa, A, n); to_mp(&xb, B, n); to_mp(&xc, C, n); to_mp(&xd, D, n); to_mp(&xe, F, n);
        mpfr_mul(&p, &xa, &xb, RNDN); mpfr_mul(&q, &xc, &xd, RNDN);
        t[0] = &p; t[1] = &q; t[2] = &xe; mpfr_sum(&r, t, 3, RNDN);
        from_mp(o, &r, n);
    }
    mpfr_clear(&xa); mpfr_clear(&xb); mpfr_clear(&xc); mpfr_clear(&xd); mpfr_clear(&xe); mpfr_clear(&p); mpfr_clear(&q); mpfr_clear(&r);
    return 0;
}

/* Precision cast: the source value exactly at its own precision, mpfr_set into the target precision
 * RNDN; a status element or a zero gives a zero with that status.  count counts components. */
int mpo_cast(int from_bits, int to_bits, const word* in, word* out, size_t count) {
    const int W = from_bits / 32, n = to_bits / 32;
    widen_range();
    mpfr_struct x, r; mpfr_init2(&x, from_bits); mpfr_init2(&r, to_bits);
    for (size_t i = 0; i < count; ++i) {
        const word* a = in + i * (size_t)(W + 3); word* o = out + i * (size_t)(n + 3);
        if (a[W + 2] || !(int32_t)a[W + 1]) { zero_num(o, n, a[W + 2]); continue; }
        to_mp(&x, a, W);
        mpfr_set(&r, &x, RNDN);
        from_mp(o, &r, n);
    }
    mpfr_clear(&x); mpfr_clear(&r);
    return 0;
}

/* ---------------------------------------------------------------- CPU baseline: MPFR multiplication chains
 * The reference's benchmark method (benchmarks/benchmark.cpp:3-94, benchmark_support.hpp:12-45): values and
 * factors are converted once into preallocated mpfr_t arrays, outside the timed region; a pass computes
 * r_i <- x_i, then r_i <- RN(r_i * f_{s,i}) for s = 0..steps-1, for every value, serially (threads = 1) or on a
 * persistent pool of `threads` workers (OpenMP), each taking one contiguous chunk.  mpo_chain_run returns the
 * pass's wall time in seconds (CLOCK_MONOTONIC); mpo_chain_result converts the last pass's values back to the
 * limb layout so they can be compared bit for bit. */
#include <time.h>
#include <omp.h>
typedef struct { int bits; size_t steps, count; mpfr_struct *x, *f, *r; } mpo_chain;

void* mpo_chain_setup(int bits, const word* x, const word* f, size_t steps, size_t count) {
    const int n = bits / 32; const size_t E = (size_t)n + 3; widen_range();
    mpo_chain* c = (mpo_chain*)calloc(1, sizeof(mpo_chain));
    c->bits = bits; c->steps = steps; c->count = count;
    c->x = (mpfr_struct*)malloc(sizeof(mpfr_struct) * count);
    c->r = (mpfr_struct*)malloc(sizeof(mpfr_struct) * count);
    c->f = (mpfr_struct*)malloc(sizeof(mpfr_struct) * count * steps);
    for (size_t i = 0; i < count; ++i) {
        mpfr_init2(&c->x[i], bits); mpfr_init2(&c->r[i], bits);
        to_mp(&c->x[i], x + i * E, n);
    }
    for (size_t k = 0; k < steps * count; ++k) { mpfr_init2(&c->f[k], bits); to_mp(&c->f[k], f + k * E, n); }
    return c;
}
double mpo_chain_run(void* h, int threads) {
    mpo_chain* c = (mpo_chain*)h;
    struct timespec t0, t1;
    clock_gettime(CLOCK_MONOTONIC, &t0);
#pragma omp parallel num_threads(threads)
    {
        widen_range();
        const size_t nt = (size_t)omp_get_num_threads(), id = (size_t)omp_get_thread_num();
        const size_t lo = c->count * id / nt, hi = c->count * (id + 1) / nt;
        for (size_t i = lo; i < hi; ++i) {
            mpfr_set(&c->r[i], &c->x[i], RNDN);
            for (size_t s = 0; s < c->steps; ++s) mpfr_mul(&c->r[i], &c->r[i], &c->f[s * c->count + i], RNDN);
        }
    }
    clock_gettime(CLOCK_MONOTONIC, &t1);
    return (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
}
void mpo_chain_result(void* h, word* out) {
    mpo_chain* c = (mpo_chain*)h;
    const int n = c->bits / 32;
    for (size_t i = 0; i < c->count; ++i) from_mp(out + i * ((size_t)n + 3), &c->r[i], n);
}
void mpo_chain_free(void* h) {
    mpo_chain* c = (mpo_chain*)h;
    for (size_t i = 0; i < c->count; ++i) { mpfr_clear(&c->x[i]); mpfr_clear(&c->r[i]); }
    for (size_t k = 0; k < c->steps * c->count; ++k) mpfr_clear(&c->f[k]);
    free(c->x); free(c->r); free(c->f); free(c);
}
