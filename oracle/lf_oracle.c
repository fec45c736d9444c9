/*
 * CPU oracle for the LimbForge batched multiprecision path.  TEST INFRASTRUCTURE ONLY:
 * nothing in the product (the limbforge_b200 package or its shared library) links, loads
 * or calls this file; tests/, __graft_entry__.smoke() and bench.py's CPU baseline use it
 * as the checker.
 *
 * This is a restatement, in plain C, of the arithmetic contract of the reference
 * (WolfNum/LimbForge include/limbforge/core.hpp and linalg.hpp::exact_dot_add), not a copy:
 * every operation is computed as an exact big integer and rounded ONCE with round to
 * nearest, ties to even.  Because each reference operation is a single correct rounding,
 * any exact method gives the same bits; the conventions that are not implied by correct
 * rounding are restated explicitly and cited:
 *
 *   element layout  Number<N> = {u32 limb[N] (little endian, top bit set when nonzero),
 *                   i32 exponent, i32 sign (-1,0,+1), u32 status}           core.hpp:23-28
 *                   value = sign * int(limb) * 2^(exponent - (32N-1))
 *   statuses        division_by_zero=1, exponent_overflow=2, invalid=4      core.hpp:22
 *                   any input status -> zero carrying the OR of the statuses core.hpp:124,138,186,318
 *   exponent range  the rounded result's exponent must lie in [-1e9, 1e9],
 *                   otherwise zero with exponent_overflow                   core.hpp:77-85
 *   zero            canonical: limbs 0, exponent 0, sign 0                  core.hpp:46-49
 *   add shortcuts   add(0,b) returns b unchanged, add(a,0) returns a;
 *                   an operand more than 32N+2 bits below returns the larger core.hpp:125-129
 *   div             b == 0 -> division_by_zero; a == 0 -> zero              core.hpp:187
 *   sqrt            negative -> invalid                                     core.hpp:218
 *   exact_dot_add   no nonzero product -> the addend itself (or zero)      linalg.hpp:281
 *
 * Sums of several exact terms (fma, dot2_add, exact dots) are rounded with the cluster
 * argument of linalg.hpp:269-273: terms sorted by magnitude are summed exactly in clusters;
 * everything after the first nonzero cluster sum S is below 2^(lsb(S)-32N-4) and only its
 * sign matters, which is the sign of the next nonzero cluster sum.
 *
 * Sequences built on these operations (complex ops, blocked Cholesky and triangular
 * solves, batched 4x4 LU, strided batched GEMM) follow the cited reference sequences.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef uint32_t word;
typedef uint64_t dword;

enum { ST_DIV0 = 1, ST_OVF = 2, ST_INVALID = 4 };
#define EMAX 1000000000LL

/* ---------------------------------------------------------------- element access */
typedef struct { word* w; int n; } num;           /* view of one element */
static inline int32_t* EXP(word* e, int n) { return (int32_t*)&e[n]; }
static inline int32_t* SGN(word* e, int n) { return (int32_t*)&e[n + 1]; }
static inline word* STS(word* e, int n) { return &e[n + 2]; }
static inline int32_t gexp(const word* e, int n) { return (int32_t)e[n]; }
static inline int32_t gsgn(const word* e, int n) { return (int32_t)e[n + 1]; }
static inline word gsts(const word* e, int n) { return e[n + 2]; }

static void set_zero(word* out, int n, word status) {
    memset(out, 0, sizeof(word) * (size_t)(n + 3));
    *STS(out, n) = status;
}
static void copy_num(word* out, const word* in, int n) { memmove(out, in, sizeof(word) * (size_t)(n + 3)); }
static void neg_copy(word* out, const word* in, int n) { copy_num(out, in, n); *SGN(out, n) = -gsgn(in, n); }

/* ---------------------------------------------------------------- big integer helpers */
static int top_bit(const word* x, int W) {           /* index of the highest set bit, -1 if zero */
    for (int i = W - 1; i >= 0; --i)
        if (x[i]) return 32 * i + 31 - __builtin_clz(x[i]);
    return -1;
}
static int get_bit(const word* x, int W, long b) {
    if (b < 0 || b >= 32L * W) return 0;
    return (x[b / 32] >> (b % 32)) & 1;
}
static word bits32(const word* x, int W, long p) {    /* 32 bits of x starting at bit p */
    word r = 0;
    if (p <= -32) return 0;
    if (p < 0) return x[0] << (-p);
    long i = p / 32; int s = (int)(p % 32);
    if (i < W) r = x[i] >> s;
    if (s && i + 1 < W) r |= x[i + 1] << (32 - s);
    return r;
}
static int any_below(const word* x, int W, long b) {  /* any set bit strictly below bit b */
    if (b <= 0) return 0;
    long whole = b / 32;
    for (long i = 0; i < whole && i < W; ++i) if (x[i]) return 1;
    if (whole < W && (b % 32) && (x[whole] & ((1u << (b % 32)) - 1))) return 1;
    return 0;
}
/* x += y << shift (x has W words, enough room) */
static void add_shifted(word* x, int W, const word* y, int Wy, long shift) {
    long ws = shift / 32; int s = (int)(shift % 32); dword c = 0;
    for (long i = 0; i + ws < W; ++i) {
        word v = 0;
        if (i < Wy) v = y[i] << s;
        if (s && i > 0 && i - 1 < Wy) v |= y[i - 1] >> (32 - s);
        if (i > Wy && !c) break;
        dword t = (dword)x[i + ws] + v + c; x[i + ws] = (word)t; c = t >> 32;
    }
}
/* x -= y << shift, two's complement in W words */
static void sub_shifted(word* x, int W, const word* y, int Wy, long shift) {
    long ws = shift / 32; int s = (int)(shift % 32); int borrow = 0;
    for (long i = 0; i + ws < W; ++i) {
        word v = 0;
        if (i < Wy) v = y[i] << s;
        if (s && i > 0 && i - 1 < Wy) v |= y[i - 1] >> (32 - s);
        if (i > Wy && !borrow) break;
        dword t = (dword)v + (dword)borrow; word old = x[i + ws];
        x[i + ws] = (word)((dword)old - t); borrow = (dword)old < t;
    }
}
static void negate_words(word* x, int W) { dword c = 1; for (int i = 0; i < W; ++i) { dword t = (dword)(word)~x[i] + c; x[i] = (word)t; c = t >> 32; } }
static int is_zero(const word* x, int W) { for (int i = 0; i < W; ++i) if (x[i]) return 0; return 1; }
static int cmp_words(const word* a, const word* b, int W) { for (int i = W - 1; i >= 0; --i) if (a[i] != b[i]) return a[i] > b[i] ? 1 : -1; return 0; }

/* ---------------------------------------------------------------- the one rounding
 * out = RN(sign * int(x) * 2^scale) to n words, or zero.  x is not modified. */
static void round_to(word* out, int n, const word* x, int W, int64_t scale, int sign, word status) {
    int h = top_bit(x, W);
    if (h < 0) { set_zero(out, n, status); return; }
    int64_t e = scale + h;
    long shift = (long)h - (32L * n - 1);              /* bit of x that becomes bit 0 of the result */
    word limb[32];
    for (int i = 0; i < n; ++i) limb[i] = bits32(x, W, shift + 32L * i);
    if (shift > 0) {
        int rb = get_bit(x, W, shift - 1);
        int st = any_below(x, W, shift - 1);
        if (rb && (st || (limb[0] & 1))) {
            int i = 0;
            while (i < n && ++limb[i] == 0) ++i;
            if (i == n) { limb[n - 1] = 0x80000000u; ++e; }
        }
    }
    if (e > EMAX || e < -EMAX) { set_zero(out, n, status | ST_OVF); return; }
    set_zero(out, n, status);
    memcpy(out, limb, sizeof(word) * (size_t)n);
    *EXP(out, n) = (int32_t)e; *SGN(out, n) = sign;
}

/* ---------------------------------------------------------------- add / sub */
static int mag_cmp(const word* a, const word* b, int n) {
    int sa = gsgn(a, n), sb = gsgn(b, n);
    if (!sa) return sb ? -1 : 0;
    if (!sb) return 1;
    if (gexp(a, n) != gexp(b, n)) return gexp(a, n) > gexp(b, n) ? 1 : -1;
    return cmp_words(a, b, n);
}
void lfo_add(int n, const word* a, const word* b, word* out) {
    word st = gsts(a, n) | gsts(b, n);
    if (st) { set_zero(out, n, st); return; }
    if (!gsgn(a, n)) { copy_num(out, b, n); return; }
    if (!gsgn(b, n)) { copy_num(out, a, n); return; }
    const word* x = a; const word* y = b;
    if (mag_cmp(a, b, n) < 0) { x = b; y = a; }
    int64_t gap = (int64_t)gexp(x, n) - gexp(y, n);
    if (gap > 32L * n + 2) { copy_num(out, x, n); return; }
    int W = 2 * n + 3; word acc[67]; memset(acc, 0, sizeof acc);
    add_shifted(acc, W, x, n, (long)gap);
    if (gsgn(x, n) == gsgn(y, n)) add_shifted(acc, W, y, n, 0);
    else sub_shifted(acc, W, y, n, 0);               /* |x| >= |y|, never negative */
    round_to(out, n, acc, W, (int64_t)gexp(y, n) - (32L * n - 1), gsgn(x, n), 0);
}
void lfo_sub(int n, const word* a, const word* b, word* out) {
    word t[35]; neg_copy(t, b, n); lfo_add(n, a, t, out);
}

/* ---------------------------------------------------------------- mul */
static void mant_mul(const word* a, const word* b, int n, word* p) {   /* p: 2n words */
    memset(p, 0, sizeof(word) * (size_t)(2 * n));
    for (int i = 0; i < n; ++i) {
        dword c = 0;
        for (int j = 0; j < n; ++j) { dword t = (dword)a[i] * b[j] + p[i + j] + c; p[i + j] = (word)t; c = t >> 32; }
        p[i + n] = (word)c;
    }
}
void lfo_mul(int n, const word* a, const word* b, word* out) {
    word st = gsts(a, n) | gsts(b, n);
    if (st || !gsgn(a, n) || !gsgn(b, n)) { set_zero(out, n, st); return; }
    word p[64]; mant_mul(a, b, n, p);
    round_to(out, n, p, 2 * n, (int64_t)gexp(a, n) + gexp(b, n) - 2 * (32L * n - 1), gsgn(a, n) * gsgn(b, n), 0);
}
void lfo_square(int n, const word* a, word* out) { lfo_mul(n, a, a, out); }

/* ---------------------------------------------------------------- div
 * q = floor(A * 2^(32n+1) / B) by binary long division; q has 32n+1 or 32n+2 bits, the
 * remainder only decides the sticky bit, appended as one extra low bit of q. */
void lfo_div(int n, const word* a, const word* b, word* out) {
    word st = gsts(a, n) | gsts(b, n);
    if (st) { set_zero(out, n, st); return; }
    if (!gsgn(b, n)) { set_zero(out, n, ST_DIV0); return; }
    if (!gsgn(a, n)) { set_zero(out, n, 0); return; }
    int W = n + 2;                                    /* remainder and divisor words */
    word r[34], d[34], q[68];
    memset(r, 0, sizeof r); memset(d, 0, sizeof d); memset(q, 0, sizeof q);
    memcpy(d, b, sizeof(word) * (size_t)n);
    long total = 32L * n + 32L * n + 1;                /* numerator bits: A then 32n+1 zeros */
    for (long i = total - 1; i >= 0; --i) {
        word carry = 0;                               /* r = 2r + bit */
        for (int k = 0; k < W; ++k) { word nv = (r[k] << 1) | carry; carry = r[k] >> 31; r[k] = nv; }
        long src = i - (32L * n + 1);
        if (src >= 0) r[0] |= get_bit(a, n, src);
        if (cmp_words(r, d, W) >= 0) { sub_shifted(r, W, d, W, 0); q[(i + 1) / 32] |= 1u << ((i + 1) % 32); }
    }
    if (!is_zero(r, W)) q[0] |= 1;                    /* sticky below the quotient */
    round_to(out, n, q, 2 * n + 2, (int64_t)gexp(a, n) - gexp(b, n) - (32L * n + 1) - 1,
             gsgn(a, n) * gsgn(b, n), 0);
}

/* ---------------------------------------------------------------- sqrt
 * Z = M * 2^t with (exponent - (32n-1) - t) even and Z of at least 64n+1 bits; the integer
 * root has at least 32n+1 bits and the sticky bit says Z is not a perfect square. */
void lfo_sqrt(int n, const word* a, word* out) {
    word st = gsts(a, n);
    if (st || !gsgn(a, n)) { set_zero(out, n, st); return; }
    if (gsgn(a, n) < 0) { set_zero(out, n, ST_INVALID); return; }
    int64_t sc = (int64_t)gexp(a, n) - (32L * n - 1);
    long t = 32L * n + 2;                              /* Z = M << t, then fix the parity */
    if ((sc - t) & 1) ++t;
    int W = 2 * n + 2;                                 /* bits of Z <= 64n + 3 */
    word Z[66], root[34], rem[68], trial[68];
    memset(Z, 0, sizeof Z); memset(root, 0, sizeof root); memset(rem, 0, sizeof rem);
    add_shifted(Z, W, a, n, t);
    int h = top_bit(Z, W); int pairs = h / 2 + 1;
    int RW = n + 2;                                    /* root words (root < 2^(33n)) */
    for (int pi = pairs - 1; pi >= 0; --pi) {
        /* rem = 4 rem + next two bits */
        word carry = 0;
        for (int k = 0; k < W; ++k) { word nv = (rem[k] << 2) | carry; carry = rem[k] >> 30; rem[k] = nv; }
        rem[0] |= (word)(get_bit(Z, W, 2L * pi) | (get_bit(Z, W, 2L * pi + 1) << 1));
        /* trial = 4 root + 1 */
        memset(trial, 0, sizeof trial);
        carry = 0;
        for (int k = 0; k < RW; ++k) { word nv = (root[k] << 2) | carry; carry = root[k] >> 30; trial[k] = nv; }
        trial[RW] = carry; trial[0] |= 1;
        /* root = 2 root */
        carry = 0;
        for (int k = 0; k < RW; ++k) { word nv = (root[k] << 1) | carry; carry = root[k] >> 31; root[k] = nv; }
        if (cmp_words(rem, trial, W) >= 0) { sub_shifted(rem, W, trial, W, 0); root[0] |= 1; }
    }
    word r2[36]; memset(r2, 0, sizeof r2);
    memcpy(r2 + 1, root, sizeof(word) * (size_t)RW);  /* shift left one word for the sticky bit */
    if (!is_zero(rem, W)) r2[0] = 1;
    round_to(out, n, r2, RW + 1, (sc - t) / 2 - 32, 1, 0);
}

/* ---------------------------------------------------------------- exact sums */
typedef struct { const word* w; int nw; int64_t scale; int sign; } term;

static int term_cmp(const void* x, const void* y) {
    const term* a = (const term*)x; const term* b = (const term*)y;
    int64_t ta = a->scale + 32L * a->nw, tb = b->scale + 32L * b->nw;
    return ta < tb ? 1 : ta > tb ? -1 : 0;
}
/* out = RN(sum of terms); the terms array is reordered.  Returns nothing; zero -> canonical. */
static void round_sum(word* out, int n, term* t, size_t count) {
    size_t m = 0;
    for (size_t i = 0; i < count; ++i) if (t[i].sign) t[m++] = t[i];
    if (!m) { set_zero(out, n, 0); return; }
    if (m <= 64) {                                   /* few terms: insertion sort, the order of term_cmp */
        for (size_t i = 1; i < m; ++i) {
            term x = t[i]; size_t j = i;
            while (j > 0 && term_cmp(&t[j - 1], &x) > 0) { t[j] = t[j - 1]; --j; }
            t[j] = x;
        }
    } else qsort(t, m, sizeof(term), term_cmp);
    int logc = 0; while (((size_t)1 << logc) < m + 1) ++logc;
    const int64_t gap = 32L * n + logc + 4;
    word* first = NULL; int first_w = 0; int64_t first_low = 0; int first_sign = 0; int follow = 0;
    for (size_t i = 0; i < m;) {
        size_t j = i + 1; int64_t low = t[i].scale, top = t[i].scale + 32L * t[i].nw;
        while (j < m && t[j].scale + 32L * t[j].nw > low - gap) { if (t[j].scale < low) low = t[j].scale; ++j; }
        int W = (int)((top - low) / 32) + 3 + (logc + 31) / 32;
        word* acc = (word*)calloc((size_t)W, sizeof(word));
        for (size_t q = i; q < j; ++q) {
            if (t[q].sign > 0) add_shifted(acc, W, t[q].w, t[q].nw, (long)(t[q].scale - low));
            else sub_shifted(acc, W, t[q].w, t[q].nw, (long)(t[q].scale - low));
        }
        int sign = 1;
        if (acc[W - 1] >> 31) { sign = -1; negate_words(acc, W); }
        if (is_zero(acc, W)) { free(acc); i = j; continue; }
        if (!first) { first = acc; first_w = W; first_low = low; first_sign = sign; i = j; continue; }
        follow = sign; free(acc); break;
    }
    if (!first) { set_zero(out, n, 0); return; }
    if (!follow) { round_to(out, n, first, first_w, first_low, first_sign, 0); free(first); return; }
    /* S * 2^D + sign(F) * 1 with D = 32n + 64: the unit lies below every rounding decision */
    const int D = 32 * n + 64;
    int W = first_w + D / 32 + 1;
    word* ext = (word*)calloc((size_t)W, sizeof(word));
    memcpy(ext + D / 32, first, sizeof(word) * (size_t)first_w);
    word one = 1;
    if (follow == first_sign) add_shifted(ext, W, &one, 1, 0); else sub_shifted(ext, W, &one, 1, 0);
    round_to(out, n, ext, W, first_low - D, first_sign, 0);
    free(ext); free(first);
}

/* RN(a*b + c) / RN(a*b - c), one rounding (mpfr_fma / mpfr_fms contract, core.hpp:317-329) */
void lfo_fma(int n, const word* a, const word* b, const word* c, int negate_c, word* out) {
    word st = gsts(a, n) | gsts(b, n) | gsts(c, n);
    if (st) { set_zero(out, n, st); return; }
    word p[64]; term t[2]; size_t k = 0;
    if (gsgn(a, n) && gsgn(b, n)) {
        mant_mul(a, b, n, p);
        t[k].w = p; t[k].nw = 2 * n; t[k].scale = (int64_t)gexp(a, n) + gexp(b, n) - 2 * (32L * n - 1);
        t[k].sign = gsgn(a, n) * gsgn(b, n); ++k;
    }
    if (gsgn(c, n)) { t[k].w = c; t[k].nw = n; t[k].scale = (int64_t)gexp(c, n) - (32L * n - 1); t[k].sign = negate_c ? -gsgn(c, n) : gsgn(c, n); ++k; }
    round_sum(out, n, t, k);
}
/* RN(a*b + c*d + e), one rounding (core.hpp:334-351) */
void lfo_dot2_add(int n, const word* a, const word* b, const word* c, const word* d, const word* e, word* out) {
    word st = gsts(a, n) | gsts(b, n) | gsts(c, n) | gsts(d, n) | gsts(e, n);
    if (st) { set_zero(out, n, st); return; }
    word p[64], q[64]; term t[3]; size_t k = 0;
    if (gsgn(a, n) && gsgn(b, n)) { mant_mul(a, b, n, p); t[k].w = p; t[k].nw = 2 * n; t[k].scale = (int64_t)gexp(a, n) + gexp(b, n) - 2 * (32L * n - 1); t[k].sign = gsgn(a, n) * gsgn(b, n); ++k; }
    if (gsgn(c, n) && gsgn(d, n)) { mant_mul(c, d, n, q); t[k].w = q; t[k].nw = 2 * n; t[k].scale = (int64_t)gexp(c, n) + gexp(d, n) - 2 * (32L * n - 1); t[k].sign = gsgn(c, n) * gsgn(d, n); ++k; }
    if (gsgn(e, n)) { t[k].w = e; t[k].nw = n; t[k].scale = (int64_t)gexp(e, n) - (32L * n - 1); t[k].sign = gsgn(e, n); ++k; }
    round_sum(out, n, t, k);
}
/* RN(c -/+ sum_k a[k*sa] * b[k*sb]) with one rounding (linalg.hpp:274-318); c may be NULL. */
void lfo_exact_dot_add(int n, const word* c, int subtract, const word* a, long sa, const word* b, long sb, size_t K, word* out) {
    const size_t E = (size_t)n + 3;
    word st = c ? gsts(c, n) : 0;
    for (size_t k = 0; k < K; ++k) st |= gsts(a + (long)k * sa * (long)E, n) | gsts(b + (long)k * sb * (long)E, n);
    if (st) { set_zero(out, n, st); return; }
    /* short dots (the factorizations' K <= block) keep their terms on the stack */
    term t_small[65]; word prod_small[64 * 64];
    const int small = K <= 64;
    term* t = small ? t_small : (term*)malloc(sizeof(term) * (K + 1));
    word* prod = small ? prod_small : (word*)malloc(sizeof(word) * (2 * (size_t)n) * (K ? K : 1));
    size_t m = 0;
    for (size_t k = 0; k < K; ++k) {
        const word* x = a + (long)k * sa * (long)E; const word* y = b + (long)k * sb * (long)E;
        if (!gsgn(x, n) || !gsgn(y, n)) continue;
        word* p = prod + 2 * (size_t)n * m;
        mant_mul(x, y, n, p);
        t[m].w = p; t[m].nw = 2 * n; t[m].scale = (int64_t)gexp(x, n) + gexp(y, n) - 2 * (32L * n - 1);
        t[m].sign = subtract ? -gsgn(x, n) * gsgn(y, n) : gsgn(x, n) * gsgn(y, n); ++m;
    }
    if (!m) {
        if (c) copy_num(out, c, n); else set_zero(out, n, 0);
        if (!small) { free(t); free(prod); }
        return;
    }
    word cc[35];
    if (c && gsgn(c, n)) { copy_num(cc, c, n); t[m].w = cc; t[m].nw = n; t[m].scale = (int64_t)gexp(c, n) - (32L * n - 1); t[m].sign = gsgn(c, n); ++m; }
    round_sum(out, n, t, m);
    if (!small) { free(t); free(prod); }
}

/* ---------------------------------------------------------------- complex (core.hpp:353-419) */
/* complex element: re then im, each n+3 words */
void lfo_cadd(int n, const word* a, const word* b, word* out) {
    const int E = n + 3; word r[35], i[35];
    lfo_add(n, a, b, r); lfo_add(n, a + E, b + E, i);
    copy_num(out, r, n); copy_num(out + E, i, n);
}
void lfo_cmul(int n, const word* a, const word* b, word* out) {
    const int E = n + 3; word p1[35], p2[35], r[35], i[35];
    lfo_mul(n, a, b, p1); lfo_mul(n, a + E, b + E, p2); lfo_sub(n, p1, p2, r);
    lfo_mul(n, a, b + E, p1); lfo_mul(n, a + E, b, p2); lfo_add(n, p1, p2, i);
    copy_num(out, r, n); copy_num(out + E, i, n);
}
void lfo_cdiv(int n, const word* a, const word* b, word* out) {
    const int E = n + 3; word p1[35], p2[35], d[35], x[35], r[35], i[35];
    lfo_mul(n, b, b, p1); lfo_mul(n, b + E, b + E, p2); lfo_add(n, p1, p2, d);
    lfo_mul(n, a, b, p1); lfo_mul(n, a + E, b + E, p2); lfo_add(n, p1, p2, x); lfo_div(n, x, d, r);
    lfo_mul(n, a + E, b, p1); lfo_mul(n, a, b + E, p2); lfo_sub(n, p1, p2, x); lfo_div(n, x, d, i);
    copy_num(out, r, n); copy_num(out + E, i, n);
}
/* cfma: re = RN(a.re b.re - a.im b.im + c.re), im = RN(a.re b.im + a.im b.re + c.im); cfms negates c */
void lfo_cfma(int n, const word* a, const word* b, const word* c, int negate_c, word* out) {
    const int E = n + 3; word m[35], cr[35], ci[35], r[35], i[35];
    neg_copy(m, a + E, n);
    if (negate_c) { neg_copy(cr, c, n); neg_copy(ci, c + E, n); } else { copy_num(cr, c, n); copy_num(ci, c + E, n); }
    lfo_dot2_add(n, a, b, m, b + E, cr, r);
    lfo_dot2_add(n, a, b + E, a + E, b, ci, i);
    copy_num(out, r, n); copy_num(out + E, i, n);
}

/* ---------------------------------------------------------------- batched element-wise driver
 * op codes follow limbforge::Operation (engine.hpp:13): add sub mul div complex_add complex_mul
 * complex_div square sqrt fma fms complex_fma complex_fms.  Broadcast index (i/stride)%period
 * (kernels.metal:7). */
static size_t bidx(size_t i, size_t stride, size_t period) { size_t j = stride > 1 ? i / stride : i; return period ? j % period : j; }
int lfo_elementwise(int bits, int op, const word* a, const word* b, const word* c, word* out, size_t count,
                    size_t bs, size_t bp, size_t cs, size_t cp) {
    if (bits < 64 || bits > 1024 || bits % 32) return 1;
    const int n = bits / 32; const size_t E = (size_t)n + 3;
    const int cx = (op >= 4 && op <= 6) || op == 11 || op == 12;
    const size_t S = cx ? 2 * E : E;
    int bad = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(|:bad)
    for (size_t i = 0; i < count; ++i) {
        const word* x = a + i * S; word* o = out + i * S;
        const word* y = b ? b + bidx(i, bs, bp) * S : NULL;
        const word* z = c ? c + bidx(i, cs, cp) * S : NULL;
        word tmp[70];
        switch (op) {
        case 0: lfo_add(n, x, y, tmp); break;
        case 1: lfo_sub(n, x, y, tmp); break;
        case 2: lfo_mul(n, x, y, tmp); break;
        case 3: lfo_div(n, x, y, tmp); break;
        case 4: lfo_cadd(n, x, y, tmp); break;
        case 5: lfo_cmul(n, x, y, tmp); break;
        case 6: lfo_cdiv(n, x, y, tmp); break;
        case 7: lfo_square(n, x, tmp); break;
        case 8: lfo_sqrt(n, x, tmp); break;
        case 9: lfo_fma(n, x, y, z, 0, tmp); break;
        case 10: lfo_fma(n, x, y, z, 1, tmp); break;
        case 11: lfo_cfma(n, x, y, z, 0, tmp); break;
        case 12: lfo_cfma(n, x, y, z, 1, tmp); break;
        default: bad = 1; continue;
        }
        memcpy(o, tmp, sizeof(word) * S);
    }
    return bad;
}
/* value <- value * f_s for s = 0..steps-1, each step rounded (the resident mul chain);
 * factors are [steps][count] */
int lfo_mul_chain(int bits, const word* x, const word* factors, size_t steps, word* out, size_t count) {
    const int n = bits / 32; const size_t E = (size_t)n + 3;
#pragma omp parallel for schedule(dynamic, 64)
    for (size_t i = 0; i < count; ++i) {
        word v[35]; copy_num(v, x + i * E, n);
        for (size_t s = 0; s < steps; ++s) { word r[35]; lfo_mul(n, v, factors + (s * count + i) * E, r); copy_num(v, r, n); }
        copy_num(out + i * E, v, n);
    }
    return 0;
}
int lfo_exact_dot_add_bits(int bits, const word* c, int subtract, const word* a, long sa, const word* b, long sb, size_t K, word* out) {
    lfo_exact_dot_add(bits / 32, c, subtract, a, sa, b, sb, K, out); return 0;
}

/* ---------------------------------------------------------------- dense products
 * C (m x nc) = op(A) B, or RN(C - op(A) B) with subtract; every entry one exact_dot_add
 * (the contract of Linalg::gemm/syrk, linalg.hpp:149-155).  Rows [r0, r1) only, so tests
 * can sample. */
int lfo_gemm_rows(int bits, int transpose_a, const word* A, const word* B, size_t m, size_t nc, size_t k,
                  word* C, int subtract, size_t r0, size_t r1) {
    const int n = bits / 32; const size_t E = (size_t)n + 3;
    if (r1 > m) r1 = m;
#pragma omp parallel for schedule(dynamic, 1)
    for (size_t i = r0; i < r1; ++i)
        for (size_t j = 0; j < nc; ++j) {
            const word* x = transpose_a ? A + i * E : A + i * k * E;
            long sx = transpose_a ? (long)m : 1;
            word* o = C + (i * nc + j) * E; word old[35]; copy_num(old, o, n);
            lfo_exact_dot_add(n, subtract ? old : NULL, subtract, x, sx, B + j * E, (long)nc, k, o);
        }
    return 0;
}
/* C (cols x cols) = A^T A (lower triangle; full when lower_only == 0; subtract requires lower) */
int lfo_syrk_rows(int bits, const word* A, size_t rows, size_t cols, word* C, int lower_only, int subtract, size_t r0, size_t r1) {
    const int n = bits / 32; const size_t E = (size_t)n + 3;
    if (r1 > cols) r1 = cols;
#pragma omp parallel for schedule(dynamic, 1)
    for (size_t i = r0; i < r1; ++i)
        for (size_t j = 0; j <= i; ++j) {
            word* o = C + (i * cols + j) * E; word old[35]; copy_num(old, o, n);
            lfo_exact_dot_add(n, subtract ? old : NULL, subtract, A + i * E, (long)cols, A + j * E, (long)cols, rows, o);
            if (!lower_only && j < i) copy_num(C + (j * cols + i) * E, o, n);
        }
    return 0;
}

/* ---------------------------------------------------------------- blocked Cholesky (linalg.mm:411-457)
 * D(c; x, y; K) = exact_dot_add(c, subtract).  Right-looking with block nb: the panel of
 * block [k0,k1) is factored row by row (l_ij = RN(D(a_ij; l_i, l_j; [k0, j)) / l_jj),
 * l_ii = sqrt(D(a_ii; l_i, l_i; [k0, i)))), then every trailing lower entry is updated by
 * one D over [k0, k1).  info[0] = pivot, info[1] = pivot sign, info[2] = pivot status. */
int lfo_cholesky(int bits, const word* A, size_t nn, word* L, size_t block, long* info) {
    const int n = bits / 32; const size_t E = (size_t)n + 3;
    size_t nb = block ? (block < nn ? block : nn) : nn;
    word* W = L;
    for (size_t i = 0; i < nn; ++i) for (size_t j = 0; j < nn; ++j) {
        if (j > i) set_zero(W + (i * nn + j) * E, n, 0); else copy_num(W + (i * nn + j) * E, A + (i * nn + j) * E, n);
    }
    info[0] = (long)nn; info[1] = 0; info[2] = 0;
#define AT(i, j) (W + ((i) * nn + (j)) * E)
    size_t p = nn;
    for (size_t k0 = 0; k0 < nn && p == nn; k0 += nb) {
        size_t k1 = k0 + nb < nn ? k0 + nb : nn;
        /* panel: diagonal block row by row */
        size_t fail = k1;
        for (size_t i = k0; i < k1 && fail == k1; ++i) {
            for (size_t j = k0; j < i; ++j) { word d[35]; lfo_exact_dot_add(n, AT(i, j), 1, AT(i, k0), 1, AT(j, k0), 1, j - k0, d); lfo_div(n, d, AT(j, j), AT(i, j)); }
            word s[35]; lfo_exact_dot_add(n, AT(i, i), 1, AT(i, k0), 1, AT(i, k0), 1, i - k0, s);
            if (gsts(s, n) || gsgn(s, n) <= 0) { fail = i; info[0] = (long)i; info[1] = gsts(s, n) ? 0 : gsgn(s, n); info[2] = (long)gsts(s, n); }
            else lfo_sqrt(n, s, AT(i, i));
        }
        size_t first = fail < k1 ? fail + 1 : k1;
        /* rows below the diagonal block are independent of one another (each reads its own row and the
           finished diagonal block), as are the entries of the trailing update: OpenMP over rows */
#pragma omp parallel for schedule(dynamic, 4)
        for (size_t i = first; i < nn; ++i)
            for (size_t j = k0; j < fail; ++j) { word d[35]; lfo_exact_dot_add(n, AT(i, j), 1, AT(i, k0), 1, AT(j, k0), 1, j - k0, d); lfo_div(n, d, AT(j, j), AT(i, j)); }
        if (fail < k1) { p = fail; break; }
        /* trailing update by block [k0, k1) */
#pragma omp parallel for schedule(dynamic, 4)
        for (size_t i = k1; i < nn; ++i)
            for (size_t j = k1; j <= i; ++j) { word d[35]; lfo_exact_dot_add(n, AT(i, j), 1, AT(i, k0), 1, AT(j, k0), 1, k1 - k0, d); copy_num(AT(i, j), d, n); }
    }
    if (p < nn) for (size_t i = p; i < nn; ++i) for (size_t j = p; j <= i; ++j) set_zero(AT(i, j), n, ST_INVALID);
#undef AT
    return 0;
}
/* Triangular solves (linalg.mm:459-488).  passes: 1 forward L X = B, 2 backward L^T X = B,
 * 3 both.  X holds B on entry (n x nrhs, row-major). */
int lfo_solve(int bits, const word* L, size_t nn, word* X, size_t nrhs, size_t block, int passes) {
    const int n = bits / 32; const size_t E = (size_t)n + 3;
    size_t nb = block ? (block < nn ? block : nn) : nn;
    if (!nn || !nrhs) return 0;
#define LL(i, j) (L + ((i) * nn + (j)) * E)
#define XX(i, c) (X + ((i) * nrhs + (c)) * E)
    if (passes & 1)
        for (size_t r0 = 0; r0 < nn; r0 += nb) {
            size_t r1 = r0 + nb < nn ? r0 + nb : nn;
#pragma omp parallel for schedule(dynamic, 1)
            for (size_t c = 0; c < nrhs; ++c)
                for (size_t i = r0; i < r1; ++i) { word d[35]; lfo_exact_dot_add(n, XX(i, c), 1, LL(i, r0), 1, XX(r0, c), (long)nrhs, i - r0, d); lfo_div(n, d, LL(i, i), XX(i, c)); }
#pragma omp parallel for schedule(dynamic, 4)
            for (size_t i = r1; i < nn; ++i)
                for (size_t c = 0; c < nrhs; ++c) { word d[35]; lfo_exact_dot_add(n, XX(i, c), 1, LL(i, r0), 1, XX(r0, c), (long)nrhs, r1 - r0, d); copy_num(XX(i, c), d, n); }
        }
    if (passes & 2)
        for (size_t r0 = (nn - 1) / nb * nb;; r0 -= nb) {
            size_t r1 = r0 + nb < nn ? r0 + nb : nn;
#pragma omp parallel for schedule(dynamic, 1)
            for (size_t c = 0; c < nrhs; ++c)
                for (size_t i = r1; i-- > r0;) {
                    word d[35];
                    if (i + 1 < r1) lfo_exact_dot_add(n, XX(i, c), 1, LL(i + 1, i), (long)nn, XX(i + 1, c), (long)nrhs, r1 - i - 1, d);
                    else copy_num(d, XX(i, c), n);
                    lfo_div(n, d, LL(i, i), XX(i, c));
                }
#pragma omp parallel for schedule(dynamic, 4)
            for (size_t i = 0; i < r0; ++i)
                for (size_t c = 0; c < nrhs; ++c) { word d[35]; lfo_exact_dot_add(n, XX(i, c), 1, LL(r0, i), (long)nn, XX(r0, c), (long)nrhs, r1 - r0, d); copy_num(XX(i, c), d, n); }
            if (!r0) break;
        }
#undef LL
#undef XX
    return 0;
}

/* ---------------------------------------------------------------- batched 4x4 complex LU (kernels.metal:210-249)
 * flags: 1 fused (cfms elimination), 2 determinant, 4 inverse.  A [count][16], B [count][4][rhs],
 * X [count][4][R] (R = 4 for the inverse), det [count], status [count]. */
static void c_minus(int n, int fused, const word* c, const word* a, const word* b, word* out) {   /* c - a*b */
    const int E = n + 3;
    if (fused) { word r[70]; lfo_cfma(n, a, b, c, 1, r); neg_copy(out, r, n); neg_copy(out + E, r + E, n); }
    else { word q[70], re[35], im[35]; lfo_cmul(n, a, b, q); lfo_sub(n, c, q, re); lfo_sub(n, c + E, q + E, im); copy_num(out, re, n); copy_num(out + E, im, n); }
}
int lfo_lu4(int bits, size_t count, unsigned rhs, int flags, const word* A, const word* B, word* X, word* det, word* status) {
    const int n = bits / 32; const int E = n + 3; const int CE = 2 * E;
    const int fused = flags & 1, want_det = flags & 2, inverse = flags & 4;
    unsigned R = inverse ? 4 : rhs;
#pragma omp parallel for schedule(dynamic, 16)
    for (size_t m = 0; m < count; ++m) {
        word a[16][70]; unsigned perm[4] = {0, 1, 2, 3}, st = 0, swaps = 0;
        for (int i = 0; i < 16; ++i) memcpy(a[i], A + (m * 16 + (size_t)i) * (size_t)CE, sizeof(word) * (size_t)CE);
        for (unsigned k = 0; k < 4 && !st; ++k) {
            unsigned piv = k;
            for (unsigned r = k + 1; r < 4; ++r) {
                const word* x = mag_cmp(a[r * 4 + k], a[r * 4 + k] + E, n) >= 0 ? a[r * 4 + k] : a[r * 4 + k] + E;
                const word* y = mag_cmp(a[piv * 4 + k], a[piv * 4 + k] + E, n) >= 0 ? a[piv * 4 + k] : a[piv * 4 + k] + E;
                if (mag_cmp(x, y, n) > 0) piv = r;
            }
            if (!gsgn(a[piv * 4 + k], n) && !gsgn(a[piv * 4 + k] + E, n)) { st = k + 1; break; }
            if (piv != k) {
                for (unsigned c = 0; c < 4; ++c) { word t[70]; memcpy(t, a[k * 4 + c], sizeof t); memcpy(a[k * 4 + c], a[piv * 4 + c], sizeof t); memcpy(a[piv * 4 + c], t, sizeof t); }
                unsigned t = perm[k]; perm[k] = perm[piv]; perm[piv] = t; ++swaps;
            }
            for (unsigned r = k + 1; r < 4; ++r) {
                word l[70]; lfo_cdiv(n, a[r * 4 + k], a[k * 4 + k], l); memcpy(a[r * 4 + k], l, sizeof l);
                for (unsigned c = k + 1; c < 4; ++c) { word v[70]; c_minus(n, fused, a[r * 4 + c], l, a[k * 4 + c], v); memcpy(a[r * 4 + c], v, sizeof v); }
            }
        }
        status[m] = st;
        if (want_det) {
            word d[70]; memset(d, 0, sizeof d);
            if (!st) {
                memcpy(d, a[0], sizeof d);
                for (int k = 1; k < 4; ++k) { word t[70]; lfo_cmul(n, d, a[k * 5], t); memcpy(d, t, sizeof d); }
                if (swaps & 1) { *SGN(d, n) = -gsgn(d, n); *SGN(d + E, n) = -gsgn(d + E, n); }
            }
            memcpy(det + m * (size_t)CE, d, sizeof(word) * (size_t)CE);
        }
        for (unsigned j = 0; j < R; ++j) {
            word y[4][70];
            for (unsigned i = 0; i < 4; ++i) {
                memset(y[i], 0, sizeof y[i]);
                if (inverse) { if (perm[i] == j) { y[i][n - 1] = 0x80000000u; *SGN(y[i], n) = 1; } }
                else memcpy(y[i], B + ((m * 4 + perm[i]) * R + j) * (size_t)CE, sizeof(word) * (size_t)CE);
            }
            if (st) {
                for (unsigned i = 0; i < 4; ++i) { word* o = X + ((m * 4 + i) * R + j) * (size_t)CE; set_zero(o, n, ST_DIV0); set_zero(o + E, n, ST_DIV0); }
                continue;
            }
            for (unsigned i = 1; i < 4; ++i) for (unsigned t = 0; t < i; ++t) { word v[70]; c_minus(n, fused, y[i], a[i * 4 + t], y[t], v); memcpy(y[i], v, sizeof v); }
            for (int i = 3; i >= 0; --i) {
                for (unsigned t = (unsigned)i + 1; t < 4; ++t) { word v[70]; c_minus(n, fused, y[i], a[i * 4 + t], y[t], v); memcpy(y[i], v, sizeof v); }
                word v[70]; lfo_cdiv(n, y[i], a[i * 5], v); memcpy(y[i], v, sizeof v);
            }
            for (unsigned i = 0; i < 4; ++i) memcpy(X + ((m * 4 + i) * R + j) * (size_t)CE, y[i], sizeof(word) * (size_t)CE);
        }
    }
    return 0;
}

/* ---------------------------------------------------------------- strided batched GEMM
 * (batched_linalg.hpp:7-14, batched_linalg.metal:16-17,24-37,145-157): C_b (+)= A_b B_b over
 * ascending k, composed (add(mul(a,b), sum) / cadd(cmul(a,b), sum)) or fused (fma / cfma),
 * negated at the end with `negative`.  Strides in elements. */
int lfo_strided_gemm(int bits, int complex_, size_t count, size_t m, size_t nc, size_t k,
                     size_t sa, size_t sb, size_t sc, int accumulate, int fused, int negative,
                     const word* A, const word* B, word* C) {
    const int n = bits / 32; const size_t E = (size_t)n + 3; const size_t S = complex_ ? 2 * E : E;
#pragma omp parallel for schedule(dynamic, 1)
    for (size_t t = 0; t < count; ++t)
        for (size_t i = 0; i < m; ++i)
            for (size_t j = 0; j < nc; ++j) {
                word sum[70]; word* o = C + (t * sc + i * nc + j) * S;
                if (accumulate) memcpy(sum, o, sizeof(word) * S); else memset(sum, 0, sizeof(word) * S);
                for (size_t q = 0; q < k; ++q) {
                    const word* x = A + (t * sa + i * k + q) * S; const word* y = B + (t * sb + q * nc + j) * S;
                    word r[70];
                    if (complex_) {
                        if (fused) lfo_cfma(n, x, y, sum, 0, r);
                        else { word p[70]; lfo_cmul(n, x, y, p); lfo_cadd(n, p, sum, r); }
                    } else {
                        if (fused) lfo_fma(n, x, y, sum, 0, r);
                        else { word p[35]; lfo_mul(n, x, y, p); lfo_add(n, p, sum, r); }
                    }
                    memcpy(sum, r, sizeof(word) * S);
                }
                if (negative) { *SGN(sum, n) = -gsgn(sum, n); if (complex_) *SGN(sum + E, n) = -gsgn(sum + E, n); }
                memcpy(o, sum, sizeof(word) * S);
            }
    return 0;
}

/* ---------------------------------------------------------------- casts and tree sums
 * Precision cast (kernels.metal:251-266): a status element or a zero becomes a zero with that status;
 * otherwise RN(sign * int(limbs) * 2^(e - (32W - 1))) at the target width; complex componentwise
 * (count counts elements; complex elements are two components). */
int lfo_cast(int from_bits, int to_bits, int complex_, const word* in, word* out, size_t count) {
    const int W = from_bits / 32, n = to_bits / 32;
    const size_t comps = count * (complex_ ? 2 : 1);
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < comps; ++i) {
        const word* src = in + i * (size_t)(W + 3);
        word* dst = out + i * (size_t)(n + 3);
        const word st = src[W + 2];
        const int32_t sign = (int32_t)src[W + 1];
        if (st || !sign) { set_zero(dst, n, st); continue; }
        round_to(dst, n, src, W, (int64_t)(int32_t)src[W] - (32LL * W - 1), sign, 0);
    }
    return 0;
}
/* Tree sum (kernels.metal:60-112): each level adds elements 2i and 2i+1 (cadd for complex), an odd
 * last element carried unrounded, until one element; an empty input sums to zero. */
int lfo_tree_sum(int bits, int complex_, const word* in, size_t count, word* out) {
    const int n = bits / 32; const size_t S = (size_t)(n + 3) * (complex_ ? 2 : 1);
    if (!count) { memset(out, 0, sizeof(word) * S); return 0; }
    word* cur = (word*)malloc(sizeof(word) * S * count);
    if (!cur) return 1;
    memcpy(cur, in, sizeof(word) * S * count);
    size_t c = count;
    while (c > 1) {
        const size_t next = (c + 1) / 2;
        for (size_t i = 0; i < next; ++i) {
            word r[70];
            if (2 * i + 1 < c) {
                if (complex_) lfo_cadd(n, cur + 2 * i * S, cur + (2 * i + 1) * S, r);
                else lfo_add(n, cur + 2 * i * S, cur + (2 * i + 1) * S, r);
            } else {
                memcpy(r, cur + 2 * i * S, sizeof(word) * S);
            }
            memcpy(cur + i * S, r, sizeof(word) * S);
        }
        c = next;
    }
    memcpy(out, cur, sizeof(word) * S);
    free(cur);
    return 0;
}

/* ---------------------------------------------------------------- segmented dots and recurrences
 * Segmented dot (kernels.metal:195-207): out[i] = the chain s <- fma(a[i*len+k], b[..], s) from s = 0 (cfma for
 * complex), b[k] when shared.  Recurrence (kernels.metal:39-58): four-value complex rings, each step
 * q = cadd(..cadd(cadd(0, cmul(w0, q0)), cmul(w1, q1)).., cmul(w3, q3)), then the ring shifts. */
int lfo_segmented_dot(int bits, int complex_, size_t segments, size_t length, int shared, const word* a, const word* b, word* out) {
    const int n = bits / 32; const size_t E = (size_t)n + 3, S = complex_ ? 2 * E : E;
#pragma omp parallel for schedule(dynamic, 16)
    for (size_t i = 0; i < segments; ++i) {
        word s[70], t[70];
        memset(s, 0, sizeof s);
        for (size_t k = 0; k < length; ++k) {
            const word* x = a + (i * length + k) * S; const word* y = b + (shared ? k : i * length + k) * S;
            if (complex_) lfo_cfma(n, x, y, s, 0, t); else lfo_fma(n, x, y, s, 0, t);
            memcpy(s, t, sizeof(word) * S);
        }
        memcpy(out + i * S, s, sizeof(word) * S);
    }
    return 0;
}
int lfo_recurrence(int bits, const word* seeds, const word* weights, word* out, size_t count, unsigned steps, unsigned spw) {
    const int n = bits / 32; const size_t S = 2 * ((size_t)n + 3);
    const size_t G = count / spw;
#pragma omp parallel for schedule(dynamic, 16)
    for (size_t i = 0; i < count; ++i) {
        word q[4][70], sum[70], p[70], t[70];
        for (int j = 0; j < 4; ++j) memcpy(q[j], seeds + ((size_t)j * count + i) * S, sizeof(word) * S);
        for (unsigned st = 0; st < steps; ++st) {
            memset(sum, 0, sizeof sum);
            for (int j = 0; j < 4; ++j) {
                lfo_cmul(n, weights + (((size_t)st * 4 + (size_t)j) * G + i / spw) * S, q[j], p);
                lfo_cadd(n, sum, p, t);
                memcpy(sum, t, sizeof(word) * S);
            }
            memcpy(q[0], q[1], sizeof q[0]); memcpy(q[1], q[2], sizeof q[1]); memcpy(q[2], q[3], sizeof q[2]);
            memcpy(q[3], sum, sizeof(word) * S);
        }
        memcpy(out + i * S, q[3], sizeof(word) * S);
    }
    return 0;
}

/* ---------------------------------------------------------------- Householder QR
 * P(x, y; K) = RN(sum x_k y_k) and D(c; x, y; K) = RN(c - sum x_k y_k), one rounding each.  Column by
 * column (the order of the reference's tests/test_qr.cpp:33-135 programs) with the dot products of the
 * reference library's blocked right-looking sequence (src/linalg.mm:488-790), so every rounding has the
 * library's term set: a block applied after its panel forms W over all rows from its first row, Y with
 * the whole block and X's update with the whole block (qr_block, linalg.mm:550-567); within a panel, a
 * column's y_i has i+1 terms and every row is reduced with all of the panel's reflectors so far
 * (linalg.mm:668-670).  The two term sets give the same values and differ only in which statuses a
 * rounding sees: when a reflector after a block's first carries a status (v scaled out of the exponent
 * range), the library gives the rows above it that status and the test's program does not; this file
 * follows the library.  Layout: A, V (m x n), R (n x n), T (blocks of nb x nb, block b at b*nb*nb, the
 * compact-WY upper triangles), tau (n), all row-major.  info: rank, reason (0 full rank, 1 zero column,
 * 2 small column, 3 status column), status, recomputed squared norms (pivoting). */
static void qr_power2(word* out, int n, int32_t e) { set_zero(out, n, 0); out[n - 1] = 0x80000000u; *EXP(out, n) = e; *SGN(out, n) = 1; }
/* x * 2^-e exactly; an exponent leaving [-1e9, 1e9] gives zero with exponent_overflow (linalg.mm:492) */
static void qr_scaled(word* out, const word* x, int n, long e) {
    if (!gsgn(x, n)) { copy_num(out, x, n); return; }
    long r = (long)gexp(x, n) - e;
    if (r > EMAX || r < -EMAX) { set_zero(out, n, gsts(x, n) | ST_OVF); return; }
    copy_num(out, x, n); *EXP(out, n) = (int32_t)r;
}
#define QP(out, a, sa, b, sb, K) lfo_exact_dot_add(n, NULL, 0, (a), (long)(sa), (b), (long)(sb), (K), (out))
#define QD(out, c, a, sa, b, sb, K) lfo_exact_dot_add(n, (c), 1, (a), (long)(sa), (b), (long)(sb), (K), (out))

/* Reflector of the reduced column x (len entries, x[0] on the diagonal, stride sx): s = P(x, x); beta = -sgn(x0) sqrt(s),
 * v0 = RN(x0 - beta), v = 2^-e (v0, x1, ...) with e = exponent(v0), tau = RN(2 / P(v, v)); nothing below the diagonal gives
 * tau = 0, v = (1, 0, ...), beta = x0.  Returns the failure reason (0 none); v is written with stride sv. */
static int qr_reflector(int n, word* x, long sx, size_t len, word* v, long sv, word* tau, int rank_bits, int* have_top,
                        long* top, word* status) {
    const size_t E = (size_t)n + 3;
    word s[35], beta[35], v0[35], pv[35];
    QP(s, x, sx, x, sx, len);
    int below = 0;
    for (size_t r = 1; r < len; ++r) below |= gsgn(x + (long)r * sx * (long)E, n) != 0;
    int reason = gsts(s, n) ? 3 : (!gsgn(x, n) && !below) ? 1 : 0;
    copy_num(beta, x, n); qr_power2(v0, n, 0);
    if (!reason && below) {
        lfo_sqrt(n, s, beta);
        if (gsgn(x, n) >= 0) *SGN(beta, n) = -gsgn(beta, n);
        lfo_sub(n, x, beta, v0);
    }
    if (!reason && rank_bits > 0 && *have_top && (long)gexp(beta, n) + rank_bits < *top) reason = 2;
    if (reason) { *status = gsts(s, n); return reason; }
    set_zero(tau, n, 0);
    if (below) {
        long e = gexp(v0, n);
        qr_scaled(v, v0, n, e);
        for (size_t r = 1; r < len; ++r) qr_scaled(v + (long)r * sv * (long)E, x + (long)r * sx * (long)E, n, e);
        word two[35]; qr_power2(two, n, 1);
        QP(pv, v, sv, v, sv, len);
        lfo_div(n, two, pv, tau);
    } else qr_power2(v, n, 0);
    copy_num(x, beta, n);
    if (!*have_top || (long)gexp(beta, n) > *top) *top = gexp(beta, n);
    *have_top = 1;
    return 0;
}
/* T column c of the block (Tb, nb x nb): T_cc = tau, T_lc = -RN(tau * P(T_l[l..c), G[l..c))) */
static void qr_t_column(int n, word* Tb, size_t nb, size_t c, const word* tau, const word* G) {
    const size_t E = (size_t)n + 3;
    copy_num(Tb + (c * nb + c) * E, tau, n);
    for (size_t l = 0; l < c; ++l) {
        word d[35], p[35];
        QP(d, Tb + (l * nb + l) * E, 1, G + l * E, 1, c - l);
        lfo_mul(n, tau, d, p);
        neg_copy(Tb + (l * nb + c) * E, p, n);
    }
}
static size_t qr_nb(size_t block, size_t nn) { return block && block < nn ? block : nn; }

int lfo_qr(int bits, const word* A, size_t m, size_t nn, size_t block, int rank_bits, word* R, word* V, word* T, word* tau, long* info) {
    const int n = bits / 32; const size_t E = (size_t)n + 3;
    const size_t nb = qr_nb(block, nn), blocks = nb ? (nn + nb - 1) / nb : 0;
    word* a = (word*)malloc(sizeof(word) * E * (m * nn + 1));
    memcpy(a, A, sizeof(word) * E * m * nn);
    memset(V, 0, sizeof(word) * E * m * nn); memset(T, 0, sizeof(word) * E * blocks * nb * nb); memset(tau, 0, sizeof(word) * E * nn);
    word* w = (word*)malloc(sizeof(word) * E * (nb + 1)); word* y = (word*)malloc(sizeof(word) * E * (nb + 1));
    word* G = (word*)malloc(sizeof(word) * E * (nb + 1));
    size_t rank = nn; int reason = 0; word status = 0; int have_top = 0; long top = 0;
#define A_(r, c) (a + ((r) * nn + (c)) * E)
#define V_(r, c) (V + ((r) * nn + (c)) * E)
    for (size_t j = 0; j < nn; ++j) {
        /* column j by the reflectors [0, min(j, rank)), block by block: an earlier block as its trailing update
           (W over rows [b0, m), Y and the update with the whole block), j's own block as its panel (w_i over rows
           [b0 + i, m), y_i with i + 1 terms, every row reduced with the q reflectors so far) */
        const size_t qn = j < rank ? j : rank, own = j / nb * nb;
        for (size_t b0 = 0; b0 < qn; b0 += nb) {
            const int panel = b0 == own;
            const size_t kb = panel ? qn - b0 : (b0 + nb < nn ? b0 + nb : nn) - b0;
            const word* Tb = T + (b0 / nb) * nb * nb * E;
#pragma omp parallel for schedule(dynamic, 1)
            for (size_t i = 0; i < kb; ++i) {
                if (panel) QP(w + i * E, V_(b0 + i, b0 + i), nn, A_(b0 + i, j), nn, m - b0 - i);
                else QP(w + i * E, V_(b0, b0 + i), nn, A_(b0, j), nn, m - b0);
            }
            for (size_t i = 0; i < kb; ++i) QP(y + i * E, Tb + i * E, nb, w, 1, panel ? i + 1 : kb);
#pragma omp parallel for schedule(dynamic, 16)
            for (size_t r = 0; r < m - b0; ++r) {
                word d[35];
                QD(d, A_(b0 + r, j), V_(b0 + r, b0), 1, y, 1, kb);
                copy_num(A_(b0 + r, j), d, n);
            }
        }
        if (rank < nn) continue;
        word t[35];
        const int why = qr_reflector(n, A_(j, j), (long)nn, m - j, V_(j, j), (long)nn, t, rank_bits, &have_top, &top, &status);
        if (why) { rank = j; reason = why; continue; }
        copy_num(tau + j * E, t, n);
        /* Gram column over the block's rows and T column */
        const size_t b0 = j / nb * nb, c = j - b0;
        word* Tb = T + (b0 / nb) * nb * nb * E;
#pragma omp parallel for schedule(dynamic, 1)
        for (size_t i = 0; i < c; ++i) QP(G + i * E, V_(b0, b0 + i), nn, V_(b0, j), nn, m - b0);
        qr_t_column(n, Tb, nb, c, t, G);
    }
    for (size_t i = 0; i < nn; ++i)
        for (size_t j = 0; j < nn; ++j) {
            if (j >= (i < rank ? i : rank)) copy_num(R + (i * nn + j) * E, A_(i, j), n);
            else set_zero(R + (i * nn + j) * E, n, 0);
        }
#undef A_
#undef V_
    info[0] = (long)rank; info[1] = reason; info[2] = (long)status; info[3] = 0;
    free(a); free(w); free(y); free(G);
    return 0;
}

/* Exact order for the pivot choice: +1 if x > y, -1 if x < y, 0 if equal; a status ranks above every value
 * (two statuses are equal) (linalg.mm:541-547) */
static int qr_compare(const word* x, const word* y, int n) {
    const word sx = gsts(x, n), sy = gsts(y, n);
    if (sx || sy) return (sx != 0) - (sy != 0);
    const int a = gsgn(x, n), b = gsgn(y, n);
    if (a != b) return a > b ? 1 : -1;
    if (!a) return 0;
    int c = gexp(x, n) != gexp(y, n) ? (gexp(x, n) > gexp(y, n) ? 1 : -1) : cmp_words(x, y, n);
    return a > 0 ? c : -c;
}
static void qr_swap(word* x, word* y, int n) { word t[35]; copy_num(t, x, n); copy_num(x, y, n); copy_num(y, t, n); }

/* Column-pivoted QR (xGEQP3 order, tests/test_qr.cpp:94-135): before step j the remaining column with the largest
 * downdated squared norm nu (status first, exact comparison, ties to the lowest original index) is swapped in;
 * column j is reduced by the block's reflectors so far (its Y entries), reflector j as unpivoted; then every
 * trailing column k gets W_jk = P(v_j, a_k) over rows [j, m), Y_jk = P(T[.][c], W_.k), r_jk = D(a_jk; V_j[block],
 * Y_.k) and nu_k = D(nu_k; r_jk, r_jk), recomputed from the reduced column when it drops to <= 0 or more than
 * bits/2 binades below its last exact value.  After the block, X = D(X; V_b, Y) with those W and Y. */
int lfo_qr_pivoted(int bits, const word* A, size_t m, size_t nn, size_t block, int rank_bits, word* R, word* V, word* T,
                   word* tau, size_t* perm, long* info) {
    const int n = bits / 32; const size_t E = (size_t)n + 3;
    const size_t nb = qr_nb(block, nn), blocks = nb ? (nn + nb - 1) / nb : 0;
    const size_t cells = m * nn + 1;
    word* a = (word*)malloc(sizeof(word) * E * cells);
    memcpy(a, A, sizeof(word) * E * m * nn);
    memset(V, 0, sizeof(word) * E * m * nn); memset(T, 0, sizeof(word) * E * blocks * nb * nb); memset(tau, 0, sizeof(word) * E * nn);
    word* nu = (word*)calloc(E * (nn + 1), sizeof(word)); word* nuref = (word*)calloc(E * (nn + 1), sizeof(word));
    word* Wr = (word*)calloc(E * (nb * nn + 1), sizeof(word)); word* Yr = (word*)calloc(E * (nb * nn + 1), sizeof(word));
    word* x = (word*)malloc(sizeof(word) * E * (m + 1)); word* G = (word*)malloc(sizeof(word) * E * (nb + 1));
    char* redo = (char*)calloc(nn + 1, 1);
    size_t rank = nn; int reason = 0; word status = 0; int have_top = 0; long top = 0; long recomputed = 0;
#define A_(r, c) (a + ((r) * nn + (c)) * E)
#define V_(r, c) (V + ((r) * nn + (c)) * E)
    for (size_t k = 0; k < nn; ++k) perm[k] = k;
#pragma omp parallel for schedule(dynamic, 1)
    for (size_t k = 0; k < nn; ++k) { QP(nu + k * E, A_(0, k), nn, A_(0, k), nn, m); copy_num(nuref + k * E, nu + k * E, n); }
    for (size_t b0 = 0; b0 < nn && rank == nn; b0 += nb) {
        const size_t kb = (b0 + nb < nn ? b0 + nb : nn) - b0;
        word* Tb = T + (b0 / nb) * nb * nb * E;
        size_t g = kb;                                   /* reflectors of this block applied after it */
        int fresh = 0;
        for (size_t c = 0; c < kb; ++c) {
            const size_t j = b0 + c;
            size_t p = j;
            for (size_t k = j + 1; k < nn; ++k) {
                const int cmp = qr_compare(nu + k * E, nu + p * E, n);
                if (cmp > 0 || (cmp == 0 && perm[k] < perm[p])) p = k;
            }
            if (p != j) {
                for (size_t r = 0; r < m; ++r) qr_swap(A_(r, j), A_(r, p), n);
                for (size_t i = 0; i < c; ++i) { qr_swap(Wr + (i * nn + j) * E, Wr + (i * nn + p) * E, n); qr_swap(Yr + (i * nn + j) * E, Yr + (i * nn + p) * E, n); }
                qr_swap(nu + j * E, nu + p * E, n); qr_swap(nuref + j * E, nuref + p * E, n);
                const size_t t = perm[j]; perm[j] = perm[p]; perm[p] = t;
            }
            for (size_t r = 0; r < m - b0; ++r) {
                if (c) QD(x + r * E, A_(b0 + r, j), V_(b0 + r, b0), 1, Yr + j * E, nn, c);
                else copy_num(x + r * E, A_(b0 + r, j), n);
            }
            word t[35];
            const int why = qr_reflector(n, x + c * E, 1, m - j, V_(j, j), (long)nn, t, rank_bits, &have_top, &top, &status);
            if (why) { rank = j; reason = why; g = c; fresh = 1; break; }
            for (size_t r = 0; r < m - b0; ++r) copy_num(A_(b0 + r, j), x + r * E, n);
            copy_num(tau + j * E, t, n);
#pragma omp parallel for schedule(dynamic, 1)
            for (size_t i = 0; i < c; ++i) QP(G + i * E, V_(b0, b0 + i), nn, V_(b0, j), nn, m - b0);
            qr_t_column(n, Tb, nb, c, t, G);
            /* trailing columns: W and Y rows c, row j of R, downdated norms */
#pragma omp parallel for schedule(dynamic, 1)
            for (size_t k = j + 1; k < nn; ++k) {
                word rj[35], d[35];
                QP(Wr + (c * nn + k) * E, V_(j, j), nn, A_(j, k), nn, m - j);
                QP(Yr + (c * nn + k) * E, Tb + c * E, nb, Wr + k * E, nn, c + 1);
                QD(rj, A_(j, k), V_(j, b0), 1, Yr + k * E, nn, c + 1);
                QD(d, nu + k * E, rj, 1, rj, 1, 1);
                copy_num(nu + k * E, d, n);
                const word* ref = nuref + k * E;
                redo[k] = gsgn(ref, n) && !gsts(ref, n) && !gsts(d, n) &&
                          (gsgn(d, n) <= 0 || (long)gexp(d, n) + 16L * n < (long)gexp(ref, n));
                if (redo[k]) {
                    const size_t len = m - j - 1;
                    word* z = (word*)malloc(sizeof(word) * E * (len + 1));
                    for (size_t i = 0; i < len; ++i) QD(z + i * E, A_(j + 1 + i, k), V_(j + 1 + i, b0), 1, Yr + k * E, nn, c + 1);
                    QP(nu + k * E, z, 1, z, 1, len);
                    copy_num(nuref + k * E, nu + k * E, n);
                    free(z);
                }
            }
            for (size_t k = j + 1; k < nn; ++k) recomputed += redo[k] != 0;
        }
        /* the block on the remaining columns, X = D(X; V_b, Y) with the whole block: with the W and Y rows formed
           during the panel, or after a failure (reflectors [b0, rank), the block's other V and T entries zero)
           with W over rows [b0, m) and Y formed afresh (linalg.mm:727-729, qr_block) */
        const size_t c0 = rank == nn ? b0 + kb : rank;
        if (g && c0 < nn && (rank == nn || fresh)) {
            if (fresh)
#pragma omp parallel for schedule(dynamic, 1)
                for (size_t k = c0; k < nn; ++k) {
                    for (size_t i = 0; i < kb; ++i) QP(Wr + (i * nn + k) * E, V_(b0, b0 + i), nn, A_(b0, k), nn, m - b0);
                    for (size_t i = 0; i < kb; ++i) QP(Yr + (i * nn + k) * E, Tb + i * E, nb, Wr + k * E, nn, kb);
                }
#pragma omp parallel for schedule(dynamic, 16)
            for (size_t r = 0; r < m - b0; ++r)
                for (size_t k = c0; k < nn; ++k) {
                    word d[35];
                    QD(d, A_(b0 + r, k), V_(b0 + r, b0), 1, Yr + k * E, nn, kb);
                    copy_num(A_(b0 + r, k), d, n);
                }
        }
    }
    for (size_t i = 0; i < nn; ++i)
        for (size_t j = 0; j < nn; ++j) {
            if (j >= (i < rank ? i : rank)) copy_num(R + (i * nn + j) * E, A_(i, j), n);
            else set_zero(R + (i * nn + j) * E, n, 0);
        }
#undef A_
#undef V_
    info[0] = (long)rank; info[1] = reason; info[2] = (long)status; info[3] = recomputed;
    free(a); free(nu); free(nuref); free(Wr); free(Yr); free(x); free(G); free(redo);
    return 0;
}

/* C (m x nrhs) <- Q^T C (qt, blocks in order) or Q C (blocks in reverse), the blocks holding reflectors [0, rank)
 * (qr_apply_n, linalg.mm:750-766; the column form is tests/test_qr.cpp:69-77) */
int lfo_qr_apply(int bits, size_t m, size_t nn, size_t block, size_t rank, const word* V, const word* T, word* C, size_t nrhs, int qt) {
    const int n = bits / 32; const size_t E = (size_t)n + 3;
    const size_t nb = qr_nb(block, nn), blocks = nb ? (rank + nb - 1) / nb : 0;
    for (size_t s = 0; s < blocks; ++s) {
        /* qr_block (linalg.mm:550-567): the whole block (V and T are zero beyond the rank), W over rows [b0, m) */
        const size_t b = qt ? s : blocks - 1 - s, b0 = b * nb, kb = (b0 + nb < nn ? b0 + nb : nn) - b0;
        const word* Tb = T + b * nb * nb * E;
#pragma omp parallel for schedule(dynamic, 1)
        for (size_t c = 0; c < nrhs; ++c) {
            word* w = (word*)malloc(sizeof(word) * E * (kb + 1)); word* y = (word*)malloc(sizeof(word) * E * (kb + 1));
            for (size_t i = 0; i < kb; ++i) QP(w + i * E, V + (b0 * nn + b0 + i) * E, nn, C + (b0 * nrhs + c) * E, nrhs, m - b0);
            for (size_t i = 0; i < kb; ++i) {
                if (qt) QP(y + i * E, Tb + i * E, nb, w, 1, kb);
                else QP(y + i * E, Tb + (i * nb) * E, 1, w, 1, kb);
            }
            for (size_t r = b0; r < m; ++r) {
                word d[35];
                QD(d, C + (r * nrhs + c) * E, V + (r * nn + b0) * E, 1, y, 1, kb);
                copy_num(C + (r * nrhs + c) * E, d, n);
            }
            free(w); free(y);
        }
    }
    return 0;
}
/* Least squares X (n x nrhs) from B (m x nrhs): Q^T B, then the blocked backward substitution with R (tests/test_qr.cpp:
 * 78-86); pivoted (perm != NULL): R[0:p,0:p] z = (Q^T b)[0:p) with blocks min(nb, p), x[perm[i]] = z_i, zero beyond p
 * (:137-147).  A rank-deficient unpivoted factor gives zero with invalid everywhere, a status column zero with invalid
 * and its status. */
int lfo_qr_solve(int bits, size_t m, size_t nn, size_t block, const long* info, const size_t* perm, const word* R,
                 const word* V, const word* T, const word* B, size_t nrhs, word* X) {
    const int n = bits / 32; const size_t E = (size_t)n + 3;
    const size_t p = (size_t)info[0];
    if (!nn || !nrhs) return 0;
    if (p < nn && (!perm || info[1] == 3)) {
        for (size_t q = 0; q < nn * nrhs; ++q) set_zero(X + q * E, n, ST_INVALID | (perm ? (word)info[2] : 0));
        return 0;
    }
    word* C = (word*)malloc(sizeof(word) * E * m * nrhs);
    memcpy(C, B, sizeof(word) * E * m * nrhs);
    lfo_qr_apply(bits, m, nn, block, p, V, T, C, nrhs, 1);
    /* the backward substitution of the upper R is the L^T pass with L = R^T */
    const size_t nb = qr_nb(block, nn) < p ? qr_nb(block, nn) : p;
    word* L = (word*)malloc(sizeof(word) * E * (p * p + 1));
    for (size_t i = 0; i < p; ++i) for (size_t j = 0; j < p; ++j) copy_num(L + (j * p + i) * E, R + (i * nn + j) * E, n);
    if (p) lfo_solve(bits, L, p, C, nrhs, nb, 2);
    for (size_t i = 0; i < nn; ++i)
        for (size_t c = 0; c < nrhs; ++c) {
            word* out = X + ((perm ? perm[i] : i) * nrhs + c) * E;
            if (i < p) copy_num(out, C + (i * nrhs + c) * E, n); else set_zero(out, n, 0);
        }
    free(C); free(L);
    return 0;
}
#undef QP
#undef QD

/* ---------------------------------------------------------------- complex Householder QR
 * The reference library's complex QR (src/linalg_complex.mm:125-306, zgeqrf convention: H = I - tau v v^H, complex
 * tau, real beta), restated right-looking as the library runs it.  Every complex dot product or update is two real
 * exact dot products over the interleaved (re, im) operand sequences, one rounding per component; the trailing
 * block updates are the real compact-WY update (qr_block, linalg.mm:550-567) of the 2 x 2-block real embeddings
 * of V and T ([[re, -im], [im, re]]) applied to the work matrix split by rows (row 2r = Re of row r, 2r + 1 = Im).
 * Complex arrays hold (re, im) element pairs.  pivot: column pivoting with real squared norms downdated by
 * |r_jk|^2 (linalg_complex.mm:160-255). */
#define CQP(out, a, sa, b, sb, K) lfo_exact_dot_add(n, NULL, 0, (a), (long)(sa), (b), (long)(sb), (K), (out))
#define CQD(out, c, a, sa, b, sb, K) lfo_exact_dot_add(n, (c), 1, (a), (long)(sa), (b), (long)(sb), (K), (out))
/* the real block update of block b on columns [c0, c1) of X (row stride ld): W = P(V_b^T X) over rows [k0, mE),
   Y = P(T_b^T W) (qt) or P(T_b W), X = D(X; V_b, Y), each with the whole block (have_y: Y given) */
static void cqr_block(int n, size_t mE, size_t nE, size_t nbE, const word* EV, const word* ET, size_t b, word* X, size_t ld,
                      size_t c0, size_t c1, int qt, word* Wb, word* Yb, int have_y) {
    const size_t E = (size_t)n + 3;
    const size_t k0 = b * nbE, kb = (k0 + nbE < nE ? k0 + nbE : nE) - k0, mr = mE - k0;
    if (c1 <= c0 || !kb) return;
    const word* Vb = EV + (k0 * nE + k0) * E; const word* Tb = ET + b * nbE * nbE * E; word* Xb = X + k0 * ld * E;
    if (!have_y) {
#pragma omp parallel for schedule(dynamic, 1)
        for (size_t j = c0; j < c1; ++j) {
            for (size_t i = 0; i < kb; ++i) CQP(Wb + (i * ld + j) * E, Vb + i * E, nE, Xb + j * E, ld, mr);
            for (size_t i = 0; i < kb; ++i) {
                if (qt) CQP(Yb + (i * ld + j) * E, Tb + i * E, nbE, Wb + j * E, ld, kb);
                else CQP(Yb + (i * ld + j) * E, Tb + i * nbE * E, 1, Wb + j * E, ld, kb);
            }
        }
    }
#pragma omp parallel for schedule(dynamic, 8)
    for (size_t r = 0; r < mr; ++r)
        for (size_t j = c0; j < c1; ++j) {
            word d[35];
            CQD(d, Xb + (r * ld + j) * E, Vb + r * nE * E, 1, Yb + j * E, ld, kb);
            copy_num(Xb + (r * ld + j) * E, d, n);
        }
}
/* the 2 x 2 real block [[re, -im], [im, re]] of z at (2r, 2c) of a real matrix with row stride ld */
static void cqr_embed(int n, word* M, size_t ld, size_t r, size_t c, const word* z) {
    const size_t E = (size_t)n + 3;
    copy_num(M + (2 * r * ld + 2 * c) * E, z, n); neg_copy(M + (2 * r * ld + 2 * c + 1) * E, z + E, n);
    copy_num(M + ((2 * r + 1) * ld + 2 * c) * E, z + E, n); copy_num(M + ((2 * r + 1) * ld + 2 * c + 1) * E, z, n);
}
static void cqr_times_i(int n, word* out, const word* z) { const size_t E = (size_t)n + 3; word t[35]; neg_copy(t, z + E, n); copy_num(out + E, z, n); copy_num(out, t, n); }
static void cqr_conj(int n, word* out, const word* z) { const size_t E = (size_t)n + 3; copy_num(out, z, n); neg_copy(out + E, z + E, n); }
static void cqr_i_conj(int n, word* out, const word* z) { const size_t E = (size_t)n + 3; word t[35]; copy_num(t, z + E, n); copy_num(out + E, z, n); copy_num(out, t, n); }

int lfo_qr_complex(int bits, const word* A, size_t m, size_t nn, size_t block, int rank_bits, int pivot, word* R, word* V, word* T,
                   word* tau, size_t* perm, long* info) {
    const int n = bits / 32; const size_t E = (size_t)n + 3, C2 = 2 * E;
    const size_t nb = qr_nb(block, nn), blocks = nb ? (nn + nb - 1) / nb : 0;
    const size_t mE = 2 * m, nE = 2 * nn, nbE = 2 * nb;
    word* Wk = (word*)calloc(E * (mE * nn + 1), sizeof(word));
    word* EV = (word*)calloc(E * (mE * nE + 1), sizeof(word));
    word* ET = (word*)calloc(E * (blocks * nbE * nbE + 1), sizeof(word));
    word* Wb = (word*)calloc(E * (nbE * nn + 1), sizeof(word)); word* Yb = (word*)calloc(E * (nbE * nn + 1), sizeof(word));
    word* Pt = (word*)calloc(C2 * (nb * m + 1), sizeof(word)); word* Vt = (word*)calloc(C2 * (nb * m + 1), sizeof(word));
    word* Vi = (word*)calloc(C2 * (nb * m + 1), sizeof(word)); word* Vr = (word*)calloc(C2 * (nb * m + 1), sizeof(word));
    word* Wp = (word*)calloc(C2 * (nb * nb + 1), sizeof(word));
    word* G = (word*)calloc(C2 * (nb + 1), sizeof(word)); word* Gc = (word*)calloc(C2 * (nb + 1), sizeof(word));
    word* Gic = (word*)calloc(C2 * (nb + 1), sizeof(word)); word* y = (word*)calloc(C2 * (nb + 1), sizeof(word));
    word* yc = (word*)calloc(C2 * (nb + 1), sizeof(word)); word* yic = (word*)calloc(C2 * (nb + 1), sizeof(word));
    word* tcol = (word*)calloc(C2 * (nb + 1), sizeof(word)); word* itcol = (word*)calloc(C2 * (nb + 1), sizeof(word));
    word* wl = (word*)calloc(C2 * (nb + 1), sizeof(word));
    word* nu = (word*)calloc(E * (nn + 1), sizeof(word)); word* nuref = (word*)calloc(E * (nn + 1), sizeof(word));
    char* flag = (char*)calloc(nn + 1, 1);
    memset(V, 0, sizeof(word) * C2 * m * nn); memset(T, 0, sizeof(word) * C2 * blocks * nb * nb); memset(tau, 0, sizeof(word) * C2 * nn);
    size_t rank = nn; int reason = 0; word status = 0; int have_top = 0; long top = 0; long recomputed = 0;
    word one[35], two[35]; qr_power2(one, n, 0); qr_power2(two, n, 1);
#define W_(r, c) (Wk + ((r) * nn + (c)) * E)
    for (size_t r = 0; r < m; ++r)
        for (size_t j = 0; j < nn; ++j) { copy_num(W_(2 * r, j), A + (r * nn + j) * C2, n); copy_num(W_(2 * r + 1, j), A + (r * nn + j) * C2 + E, n); }
    for (size_t k = 0; k < nn; ++k) perm[k] = k;
    if (pivot)
#pragma omp parallel for schedule(dynamic, 1)
        for (size_t k = 0; k < nn; ++k) { CQP(nu + k * E, W_(0, k), nn, W_(0, k), nn, mE); copy_num(nuref + k * E, nu + k * E, n); }
    size_t failed_done = 0;
    for (size_t k0 = 0, first = 1; k0 < nn; first = 0) {
        const size_t k1 = k0 + nb < nn ? k0 + nb : nn, kb = k1 - k0, mr = m - k0, b = k0 / nb;
        word* Tb = T + b * nb * nb * C2;
        (void)first;
        /* ---- panel [k0, k1) */
        for (size_t c = 0; c < kb; ++c) {
            if (!pivot)
                for (size_t r = 0; r < mr; ++r) { copy_num(Pt + (c * mr + r) * C2, W_(2 * (k0 + r), k0 + c), n); copy_num(Pt + (c * mr + r) * C2 + E, W_(2 * (k0 + r) + 1, k0 + c), n); }
        }
        memset(Vt, 0, sizeof(word) * C2 * kb * mr); memset(Vi, 0, sizeof(word) * C2 * kb * mr); memset(Vr, 0, sizeof(word) * C2 * mr * nb);
        size_t done = kb;
        for (size_t c = 0; c < kb; ++c) {
            const size_t j = k0 + c;
            word* x = Pt + c * mr * C2;
            if (pivot) {
                size_t p = j;
                for (size_t k = j + 1; k < nn; ++k) { const int cmp = qr_compare(nu + k * E, nu + p * E, n); if (cmp > 0 || (cmp == 0 && perm[k] < perm[p])) p = k; }
                if (p != j) {
                    for (size_t r = 0; r < mE; ++r) qr_swap(W_(r, j), W_(r, p), n);
                    for (size_t i = 0; i < 2 * c; ++i) { qr_swap(Wb + (i * nn + j) * E, Wb + (i * nn + p) * E, n); qr_swap(Yb + (i * nn + j) * E, Yb + (i * nn + p) * E, n); }
                    qr_swap(nu + j * E, nu + p * E, n); qr_swap(nuref + j * E, nuref + p * E, n);
                    const size_t t = perm[j]; perm[j] = perm[p]; perm[p] = t;
                }
                for (size_t r = 0; r < mr; ++r) { copy_num(x + r * C2, W_(2 * (k0 + r), j), n); copy_num(x + r * C2 + E, W_(2 * (k0 + r) + 1, j), n); }
            }
            const size_t q = (j < rank ? j : rank) - k0;
            const int reflect = rank == nn;
            for (size_t i = 0; i < q; ++i) {
                if (pivot) { copy_num(y + i * C2, Yb + (2 * i * nn + j) * E, n); copy_num(y + i * C2 + E, Yb + ((2 * i + 1) * nn + j) * E, n); }
                else {
                    for (size_t l = 0; l <= i; ++l) { memcpy(tcol + l * C2, Tb + (l * nb + i) * C2, sizeof(word) * C2); cqr_times_i(n, itcol + l * C2, tcol + l * C2); memcpy(wl + l * C2, Wp + (l * nb + c) * C2, sizeof(word) * C2); }
                    CQP(y + i * C2, tcol, 1, wl, 1, 2 * (i + 1)); CQP(y + i * C2 + E, itcol, 1, wl, 1, 2 * (i + 1));
                }
                cqr_conj(n, yc + i * C2, y + i * C2); cqr_i_conj(n, yic + i * C2, y + i * C2);
            }
            if (q)
#pragma omp parallel for schedule(dynamic, 16)
                for (size_t r = 0; r < mr; ++r) {
                    word d[35];
                    CQD(d, x + r * C2, Vr + r * nb * C2, 1, yc, 1, 2 * q); copy_num(x + r * C2, d, n);
                    CQD(d, x + r * C2 + E, Vr + r * nb * C2, 1, yic, 1, 2 * q); copy_num(x + r * C2 + E, d, n);
                }
            if (!reflect) continue;
            word* xc = x + c * C2; const size_t len = mr - c;
            word s[35], beta[35], v0[35];
            CQP(s, xc, 1, xc, 1, 2 * len);
            int below = 0;
            for (size_t r = 1; r < len; ++r) below |= gsgn(xc + r * C2, n) != 0 || gsgn(xc + r * C2 + E, n) != 0;
            const int needs = below || gsgn(xc + E, n) != 0;
            int why = gsts(s, n) ? 3 : (!gsgn(xc, n) && !gsgn(xc + E, n) && !below) ? 1 : 0;
            copy_num(beta, xc, n); copy_num(v0, one, n);
            if (!why && needs) { lfo_sqrt(n, s, beta); if (gsgn(xc, n) >= 0) *SGN(beta, n) = -gsgn(beta, n); lfo_sub(n, xc, beta, v0); }
            if (!why && rank_bits > 0 && have_top && (long)gexp(beta, n) + rank_bits < top) why = 2;
            if (why) { rank = j; reason = why; status = gsts(s, n); if (pivot) { done = c; break; } continue; }
            word* vc = Vt + c * mr * C2; word* ic = Vi + c * mr * C2;
            word tj[70]; memset(tj, 0, sizeof tj);
            if (needs) {
                const long e = gexp(v0, n);
                qr_scaled(vc + c * C2, v0, n, e); qr_scaled(vc + c * C2 + E, xc + E, n, e);
                for (size_t r = c + 1; r < mr; ++r) { qr_scaled(vc + r * C2, x + r * C2, n, e); qr_scaled(vc + r * C2 + E, x + r * C2 + E, n, e); }
                word sv[35];
                CQP(sv, vc + c * C2, 1, vc + c * C2, 1, 2 * len);
                const word* vim = vc + c * C2 + E;
                if (!gsgn(vim, n) && !gsts(vim, n)) lfo_div(n, two, sv, tj);
                else {
                    word a[35], sb[35], bb[35], d[35], z[35], t2[35];
                    qr_scaled(a, sv, n, 1); qr_scaled(sb, beta, n, e); lfo_mul(n, sb, vim, bb);
                    set_zero(z, n, 0); lfo_dot2_add(n, a, a, bb, bb, z, d);
                    lfo_div(n, a, d, tj); lfo_div(n, bb, d, t2); neg_copy(tj + E, t2, n);
                }
            } else { copy_num(vc + c * C2, one, n); set_zero(vc + c * C2 + E, n, 0); }
            copy_num(xc, beta, n); set_zero(xc + E, n, 0);
            memcpy(tau + j * C2, tj, sizeof(word) * C2);
            if (!have_top || (long)gexp(beta, n) > top) top = gexp(beta, n);
            have_top = 1;
            for (size_t r = c; r < mr; ++r) { cqr_times_i(n, ic + r * C2, vc + r * C2); memcpy(Vr + (r * nb + c) * C2, vc + r * C2, sizeof(word) * C2); }
            /* Gram column and (unpivoted) the panel W row c */
            const size_t ndots = pivot ? c : kb - 1;
#pragma omp parallel for schedule(dynamic, 1)
            for (size_t u = 0; u < ndots; ++u) {
                if (u < c) {
                    CQP(G + u * C2, Vt + (u * mr + c) * C2, 1, vc + c * C2, 1, 2 * len);
                    CQP(G + u * C2 + E, Vi + (u * mr + c) * C2, 1, vc + c * C2, 1, 2 * len);
                } else {
                    CQP(Wp + (c * nb + u + 1) * C2, vc + c * C2, 1, Pt + ((u + 1) * mr + c) * C2, 1, 2 * len);
                    CQP(Wp + (c * nb + u + 1) * C2 + E, ic + c * C2, 1, Pt + ((u + 1) * mr + c) * C2, 1, 2 * len);
                }
            }
            if (pivot)
#pragma omp parallel for schedule(dynamic, 1)
                for (size_t k = j + 1; k < nn; ++k) {
                    CQP(Wb + (2 * c * nn + k) * E, vc + c * C2, 1, W_(2 * (k0 + c), k), nn, 2 * len);
                    CQP(Wb + ((2 * c + 1) * nn + k) * E, ic + c * C2, 1, W_(2 * (k0 + c), k), nn, 2 * len);
                }
            /* T column: T_cc = tau, T_lc = -RN(tau * P(T_b[l][l..c) . G[l..c))) per component */
            for (size_t l = 0; l < c; ++l) { cqr_conj(n, Gc + l * C2, G + l * C2); cqr_i_conj(n, Gic + l * C2, G + l * C2); }
            memcpy(Tb + (c * nb + c) * C2, tj, sizeof(word) * C2);
            for (size_t l = 0; l < c; ++l) {
                word p[70], z[70], zero2[70];
                CQP(p, Tb + (l * nb + l) * C2, 1, Gc + l * C2, 1, 2 * (c - l));
                CQP(p + E, Tb + (l * nb + l) * C2, 1, Gic + l * C2, 1, 2 * (c - l));
                memset(zero2, 0, sizeof zero2);
                lfo_cfma(n, tj, p, zero2, 0, z);
                neg_copy(Tb + (l * nb + c) * C2, z, n); neg_copy(Tb + (l * nb + c) * C2 + E, z + E, n);
            }
            if (pivot && j + 1 < nn) {
                for (size_t l = 0; l <= c; ++l) { memcpy(tcol + l * C2, Tb + (l * nb + c) * C2, sizeof(word) * C2); cqr_times_i(n, itcol + l * C2, tcol + l * C2); }
#pragma omp parallel for schedule(dynamic, 1)
                for (size_t k = j + 1; k < nn; ++k) {
                    word* yk = (word*)malloc(sizeof(word) * C2 * (c + 1)); word* yik = (word*)malloc(sizeof(word) * C2 * (c + 1));
                    CQP(Yb + (2 * c * nn + k) * E, tcol, 1, Wb + k * E, nn, 2 * (c + 1));
                    CQP(Yb + ((2 * c + 1) * nn + k) * E, itcol, 1, Wb + k * E, nn, 2 * (c + 1));
                    for (size_t l = 0; l <= c; ++l) {
                        word z[70]; copy_num(z, Yb + (2 * l * nn + k) * E, n); copy_num(z + E, Yb + ((2 * l + 1) * nn + k) * E, n);
                        cqr_conj(n, yk + l * C2, z); cqr_i_conj(n, yik + l * C2, z);
                    }
                    word rj[70], d[35];
                    CQD(rj, W_(2 * j, k), Vr + c * nb * C2, 1, yk, 1, 2 * (c + 1));
                    CQD(rj + E, W_(2 * j + 1, k), Vr + c * nb * C2, 1, yik, 1, 2 * (c + 1));
                    CQD(d, nu + k * E, rj, 1, rj, 1, 2);
                    copy_num(nu + k * E, d, n);
                    const word* ref = nuref + k * E;
                    flag[k] = gsgn(ref, n) && !gsts(ref, n) && !gsts(d, n) && (gsgn(d, n) <= 0 || (long)gexp(d, n) + 16L * n < (long)gexp(ref, n));
                    if (flag[k]) {
                        const size_t zl = m - j - 1;
                        word* z = (word*)malloc(sizeof(word) * C2 * (zl + 1));
                        for (size_t r = j + 1; r < m; ++r) {
                            CQD(z + (r - j - 1) * C2, W_(2 * r, k), Vr + (r - k0) * nb * C2, 1, yk, 1, 2 * (c + 1));
                            CQD(z + (r - j - 1) * C2 + E, W_(2 * r + 1, k), Vr + (r - k0) * nb * C2, 1, yik, 1, 2 * (c + 1));
                        }
                        CQP(nu + k * E, z, 1, z, 1, 2 * zl);
                        copy_num(nuref + k * E, nu + k * E, n);
                        free(z);
                    }
                    free(yk); free(yik);
                }
                for (size_t k = j + 1; k < nn; ++k) recomputed += flag[k] != 0;
            }
        }
        /* write back the panel (R entries and remainders), V and its embedding, and the embedding of T_b */
        for (size_t r = 0; r < mr; ++r)
            for (size_t c = 0; c < done; ++c) {
                const word* xv = Pt + (c * mr + r) * C2; const word* vv = Vt + (c * mr + r) * C2;
                copy_num(W_(2 * (k0 + r), k0 + c), xv, n); copy_num(W_(2 * (k0 + r) + 1, k0 + c), xv + E, n);
                memcpy(V + ((k0 + r) * nn + k0 + c) * C2, vv, sizeof(word) * C2);
                cqr_embed(n, EV, nE, k0 + r, k0 + c, vv);
            }
        word* Eb = ET + b * nbE * nbE * E;
        for (size_t l = 0; l < kb; ++l) for (size_t c = l; c < kb; ++c) cqr_embed(n, Eb, nbE, l, c, Tb + (l * nb + c) * C2);
        const size_t p = k1 < rank ? k1 : rank;
        /* the block on the trailing columns (one update of columns [k1, n) gives the bits of the look-ahead split) */
        if (pivot) {
            if (p < k1) { if (p > k0) cqr_block(n, mE, nE, nbE, EV, ET, b, Wk, nn, p, nn, 1, Wb, Yb, 0); break; }
            if (k1 < nn) cqr_block(n, mE, nE, nbE, EV, ET, b, Wk, nn, k1, nn, 1, Wb, Yb, 1);
        } else {
            if (p < k1) { if (p > k0 && k1 < nn) cqr_block(n, mE, nE, nbE, EV, ET, b, Wk, nn, k1, nn, 1, Wb, Yb, 0); break; }
            if (k1 < nn) cqr_block(n, mE, nE, nbE, EV, ET, b, Wk, nn, k1, nn, 1, Wb, Yb, 0);
        }
        k0 = k1;
        failed_done = done;
    }
    (void)failed_done;
    for (size_t i = 0; i < nn; ++i)
        for (size_t j = 0; j < nn; ++j) {
            word* out = R + (i * nn + j) * C2;
            if (j >= (i < rank ? i : rank)) { copy_num(out, W_(2 * i, j), n); copy_num(out + E, W_(2 * i + 1, j), n); }
            else { set_zero(out, n, 0); set_zero(out + E, n, 0); }
        }
#undef W_
    info[0] = (long)rank; info[1] = reason; info[2] = (long)status; info[3] = recomputed;
    free(Wk); free(EV); free(ET); free(Wb); free(Yb); free(Pt); free(Vt); free(Vi); free(Vr); free(Wp); free(G); free(Gc); free(Gic);
    free(y); free(yc); free(yic); free(tcol); free(itcol); free(wl); free(nu); free(nuref); free(flag);
    return 0;
}
static void cqr_embeddings(int n, size_t m, size_t nn, size_t nb, const word* V, const word* T, word* EV, word* ET) {
    const size_t E = (size_t)n + 3, C2 = 2 * E, blocks = nb ? (nn + nb - 1) / nb : 0;
    for (size_t r = 0; r < m; ++r) for (size_t c = 0; c < nn; ++c) cqr_embed(n, EV, 2 * nn, r, c, V + (r * nn + c) * C2);
    for (size_t b = 0; b < blocks; ++b)
        for (size_t l = 0; l < nb; ++l) for (size_t c = l; c < nb; ++c) cqr_embed(n, ET + b * 4 * nb * nb * E, 2 * nb, l, c, T + (b * nb * nb + l * nb + c) * C2);
    (void)C2;
}
/* B (m x nrhs complex) <- Q^H B (adjoint, blocks in order) or Q B (reverse) over the blocks holding reflectors [0, rank):
 * the real block updates of the embeddings on B split by rows (linalg_complex.mm:311-325) */
int lfo_qr_complex_apply(int bits, size_t m, size_t nn, size_t block, size_t rank, const word* V, const word* T, word* B, size_t nrhs, int adjoint) {
    const int n = bits / 32; const size_t E = (size_t)n + 3, C2 = 2 * E;
    const size_t nb = qr_nb(block, nn), blocks = nb ? (rank + nb - 1) / nb : 0, nblk = nb ? (nn + nb - 1) / nb : 0;
    if (!blocks || !nrhs || !m) return 0;
    word* EV = (word*)calloc(E * (4 * m * nn + 1), sizeof(word)); word* ET = (word*)calloc(E * (4 * nblk * nb * nb + 1), sizeof(word));
    word* W = (word*)calloc(E * (2 * m * nrhs + 1), sizeof(word));
    word* Wb = (word*)calloc(E * (2 * nb * nrhs + 1), sizeof(word)); word* Yb = (word*)calloc(E * (2 * nb * nrhs + 1), sizeof(word));
    cqr_embeddings(n, m, nn, nb, V, T, EV, ET);
    for (size_t r = 0; r < m; ++r) for (size_t c = 0; c < nrhs; ++c) { copy_num(W + (2 * r * nrhs + c) * E, B + (r * nrhs + c) * C2, n); copy_num(W + ((2 * r + 1) * nrhs + c) * E, B + (r * nrhs + c) * C2 + E, n); }
    for (size_t q = 0; q < blocks; ++q) cqr_block(n, 2 * m, 2 * nn, 2 * nb, EV, ET, adjoint ? q : blocks - 1 - q, W, nrhs, 0, nrhs, adjoint, Wb, Yb, 0);
    for (size_t r = 0; r < m; ++r) for (size_t c = 0; c < nrhs; ++c) { copy_num(B + (r * nrhs + c) * C2, W + (2 * r * nrhs + c) * E, n); copy_num(B + (r * nrhs + c) * C2 + E, W + ((2 * r + 1) * nrhs + c) * E, n); }
    free(EV); free(ET); free(W); free(Wb); free(Yb);
    return 0;
}
/* X = R^-1 (Q^H B)[0, n): the real backward substitution on the embedding of R (blocks 2 min(nb, p)); pivoted: the leading
 * 2p x 2p block, x[perm[i]] = z_i, zero beyond p; rank-deficient unpivoted or a status column: invalid zeros
 * (linalg_complex.mm:331-345) */
int lfo_qr_complex_solve(int bits, size_t m, size_t nn, size_t block, const long* info, const size_t* perm, const word* R,
                         const word* V, const word* T, const word* B, size_t nrhs, word* X) {
    const int n = bits / 32; const size_t E = (size_t)n + 3, C2 = 2 * E;
    const size_t p = (size_t)info[0];
    if (!nn || !nrhs) return 0;
    if (p < nn && (!perm || info[1] == 3)) {
        for (size_t q = 0; q < nn * nrhs; ++q) { set_zero(X + q * C2, n, ST_INVALID | (perm ? (word)info[2] : 0)); set_zero(X + q * C2 + E, n, ST_INVALID | (perm ? (word)info[2] : 0)); }
        return 0;
    }
    word* C = (word*)malloc(sizeof(word) * C2 * (m * nrhs + 1));
    memcpy(C, B, sizeof(word) * C2 * m * nrhs);
    lfo_qr_complex_apply(bits, m, nn, block, p, V, T, C, nrhs, 1);
    const size_t nb = qr_nb(block, nn), P2 = 2 * p;
    word* L = (word*)calloc(E * (P2 * P2 + 1), sizeof(word));      /* transpose of the leading 2p x 2p block of R's embedding */
    word* Cs = (word*)calloc(E * (P2 * nrhs + 1), sizeof(word));
    word* ER = (word*)calloc(E * (4 * p * p + 1), sizeof(word));
    for (size_t i = 0; i < p; ++i) for (size_t j = 0; j < p; ++j) cqr_embed(n, ER, P2, i, j, R + (i * nn + j) * C2);
    for (size_t i = 0; i < P2; ++i) for (size_t j = 0; j < P2; ++j) copy_num(L + (j * P2 + i) * E, ER + (i * P2 + j) * E, n);
    for (size_t i = 0; i < p; ++i) for (size_t c = 0; c < nrhs; ++c) { copy_num(Cs + (2 * i * nrhs + c) * E, C + (i * nrhs + c) * C2, n); copy_num(Cs + ((2 * i + 1) * nrhs + c) * E, C + (i * nrhs + c) * C2 + E, n); }
    if (p) lfo_solve(bits, L, P2, Cs, nrhs, 2 * (nb < p ? nb : p), 2);
    for (size_t i = 0; i < nn; ++i)
        for (size_t c = 0; c < nrhs; ++c) {
            word* out = X + ((perm ? perm[i] : i) * nrhs + c) * C2;
            if (i < p) { copy_num(out, Cs + (2 * i * nrhs + c) * E, n); copy_num(out + E, Cs + ((2 * i + 1) * nrhs + c) * E, n); }
            else { set_zero(out, n, 0); set_zero(out + E, n, 0); }
        }
    free(C); free(L); free(Cs); free(ER);
    return 0;
}
#undef CQP
#undef CQD

/* ---------------------------------------------------------------- exact batched 4 x 4 products
 * The exact 4 x 4 batch of the reference's experiment (benchmarks/experiments/exact_gemm4/README.md, prototype.hpp:
 * 5-24): fixed row-major 4 x 4 matrices, matrix t at A + t*sa, B + t*sb, C + t*sc elements (stride 0 broadcasts an
 * input); each real output component is RN(C_old + sum_k a_ik b_kj), one rounding of the exact sum (C_old left out
 * without accumulation), then negated when asked; a complex component sums its eight signed real products.
 * Statuses: zero with the OR of every operand the component reads (and C_old); no nonzero product gives C_old (or
 * zero); exact cancellation gives canonical zero. */
int lfo_exact_gemm4(int bits, int complex_, size_t count, size_t sa, size_t sb, size_t sc, int accumulate, int negative,
                    const word* A, const word* B, word* C) {
    const int n = bits / 32; const size_t E = (size_t)n + 3, S = complex_ ? 2 * E : E;
#pragma omp parallel for schedule(static)
    for (size_t t = 0; t < count; ++t)
        for (size_t i = 0; i < 4; ++i)
            for (size_t j = 0; j < 4; ++j) {
                word* out = C + (t * sc + i * 4 + j) * S;
                const word* a = A + (t * sa + i * 4) * S;
                const word* b = B + (t * sb + j) * S;
                if (!complex_) {
                    word r[35];
                    lfo_exact_dot_add(n, accumulate ? out : NULL, 0, a, 1, b, 4, 4, r);
                    if (negative) *SGN(r, n) = -gsgn(r, n);
                    copy_num(out, r, n);
                } else {
                    /* re: a.re b.re - a.im b.im; im: a.re b.im + a.im b.re, over the interleaved (re, im) sequence of row i */
                    word br[8 * 35], bi[8 * 35], r[35], q[35];
                    for (int k = 0; k < 4; ++k) {
                        const word* z = b + (size_t)k * 4 * S;
                        copy_num(br + (2 * k) * E, z, n); neg_copy(br + (2 * k + 1) * E, z + E, n);
                        copy_num(bi + (2 * k) * E, z + E, n); copy_num(bi + (2 * k + 1) * E, z, n);
                    }
                    lfo_exact_dot_add(n, accumulate ? out : NULL, 0, a, 1, br, 1, 8, r);
                    lfo_exact_dot_add(n, accumulate ? out + E : NULL, 0, a, 1, bi, 1, 8, q);
                    if (negative) { *SGN(r, n) = -gsgn(r, n); *SGN(q, n) = -gsgn(q, n); }
                    copy_num(out, r, n); copy_num(out + E, q, n);
                }
            }
    return 0;
}
