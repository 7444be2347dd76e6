/*
 * gf_oracle.c -- CPU ORACLE (test infrastructure only; never part of the product path).
 *
 * A plain-C restatement of genefer's bit-exact integer transform
 * `transformCPUi32` (src/transformCPUi32.h) and of the residue utilities in
 * `gint` (src/gint.h).  Only tests/, __graft_entry__.smoke() and the CPU
 * baseline leg of bench.py load this library, and only as the checker.
 *
 * The restatement keeps the reference's data layout and operation order so
 * that the raw RNS state after every call equals the reference's bit for bit:
 *   - three 32-bit NTT primes, 4 interleaved lanes per element
 *     (src/transformCPUi32.h:19-25, 115-131);
 *   - digit i lives in lane i / (N/4), element i % (N/4) (getZi, :800-810);
 *   - forward0 / recursive square / backward0 / baseMod (:619-772, :857-868).
 * Modular products are canonical residues in [0, p), so computing them with
 * `%` by a compile-time prime gives exactly the values the reference's
 * p_inv-based product (:149-166) gives.  The reference's Barrett division
 * (:427-480) is an exact truncated division within its input range; here the
 * same quotient/remainder come from 128-bit integer division.
 *
 * Pinned by tests/test_oracle.py against the residues quoted in the
 * reference's own sources (src/main.cpp:409-443, design/rns.cpp:596-603) and
 * against the reference transform itself (oracle/_ref, built from the
 * reference sources by oracle/Makefile).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define GFO_API __attribute__((visibility("default")))

/* src/transformCPUi32.h:19-21 and :84-86 (primes and primitive roots). */
#define P1 4194304001u /* 125 * 2^25 + 1, root 3 */
#define P2 4076863489u /* 243 * 2^24 + 1, root 7 */
#define P3 3942645761u /* 235 * 2^24 + 1, root 3 */

typedef unsigned __int128 u128;
typedef __int128 i128;

static inline uint32_t modp(int k) { return (k == 0) ? P1 : ((k == 1) ? P2 : P3); }

/* Zp::operator+ / operator- / operator* (src/transformCPUi32.h:43-58). */
static inline uint32_t add_p(uint32_t a, uint32_t b, uint32_t p) { return (a >= p - b) ? a + b - p : a + b; }
static inline uint32_t sub_p(uint32_t a, uint32_t b, uint32_t p) { return (a < b) ? a - b + p : a - b; }
static inline uint32_t mul1(uint32_t a, uint32_t b) { return (uint32_t)(((uint64_t)a * b) % P1); }
static inline uint32_t mul2(uint32_t a, uint32_t b) { return (uint32_t)(((uint64_t)a * b) % P2); }
static inline uint32_t mul3(uint32_t a, uint32_t b) { return (uint32_t)(((uint64_t)a * b) % P3); }
static inline uint32_t mul_p(uint32_t a, uint32_t b, int k)
{
	return (k == 0) ? mul1(a, b) : ((k == 1) ? mul2(a, b) : mul3(a, b));
}
static inline uint32_t neg_p(uint32_t a, uint32_t p) { return (a != 0) ? p - a : 0; }
/* Zp(int32) constructor and Zp::getInt (:36, :39). */
static inline uint32_t from_int(int32_t i, uint32_t p) { return (i < 0) ? p - (uint32_t)(-(int64_t)i) : (uint32_t)i; }
static inline int32_t to_int(uint32_t n, uint32_t p) { return (n > p / 2) ? (int32_t)(n - p) : (int32_t)n; }

/* Zp::pow (:64-77). */
static uint32_t pow_p(uint32_t x, uint64_t e, int k)
{
	uint32_t r = 1, y = x;
	if (e == 0) return 1;
	for (uint64_t i = e; i > 1; i /= 2) { if (i % 2 != 0) r = mul_p(r, y, k); y = mul_p(y, y, k); }
	return mul_p(r, y, k);
}
static const uint32_t g_root[3] = { 3, 7, 3 };
/* Zp::prRoot_n (:80). */
static uint32_t prroot_n(uint64_t n, int k) { return pow_p(g_root[k], (modp(k) - 1) / n, k); }

/* transform::bitRev (src/transform.h:105-110). */
static size_t bitrev(size_t i, size_t n)
{
	size_t r = 0;
	for (size_t k = n, j = i; k > 1; k /= 2, j /= 2) r = (2 * r) | (j % 2);
	return r;
}

/* RNS4: 3 primes x 4 lanes (:191-232). */
typedef struct { uint32_t r[3][4]; } rns4;

static inline rns4 r4_add(const rns4 *a, const rns4 *b)
{
	rns4 o;
	for (int k = 0; k < 3; ++k) for (int l = 0; l < 4; ++l) o.r[k][l] = add_p(a->r[k][l], b->r[k][l], modp(k));
	return o;
}
static inline rns4 r4_sub(const rns4 *a, const rns4 *b)
{
	rns4 o;
	for (int k = 0; k < 3; ++k) for (int l = 0; l < 4; ++l) o.r[k][l] = sub_p(a->r[k][l], b->r[k][l], modp(k));
	return o;
}
static inline rns4 r4_mul(const rns4 *a, const rns4 *b)
{
	rns4 o;
	for (int l = 0; l < 4; ++l) o.r[0][l] = mul1(a->r[0][l], b->r[0][l]);
	for (int l = 0; l < 4; ++l) o.r[1][l] = mul2(a->r[1][l], b->r[1][l]);
	for (int l = 0; l < 4; ++l) o.r[2][l] = mul3(a->r[2][l], b->r[2][l]);
	return o;
}

typedef struct
{
	uint32_t b, n;
	size_t size, size_4, num_regs;
	uint32_t norm[3];      /* Zp::norm(2^(n-1)) (:508, :79) */
	uint32_t w0[3][3];     /* forward0 roots w1,w2,w3 per prime (:621-623) */
	uint32_t wi0[3][3];    /* backward0 roots wi1,wi2,wi3 (:629-631) */
	rns4 *z;               /* num_regs registers of size_4 elements */
	rns4 *wr;              /* 2 * size_4: forward then inverse roots (:511, :514-540) */
	rns4 *zp;              /* multiplicand (:512) */
} gfo_t;

/* Constructor twiddles (src/transformCPUi32.h:514-540). */
static void build_roots(gfo_t *t)
{
	const size_t size_4 = t->size_4;
	rns4 *const wr = t->wr, *const wri = &t->wr[size_4];
	memset(wr, 0, 2 * size_4 * sizeof(rns4));
	for (size_t s_4 = 1; s_4 < size_4 / 2; s_4 *= 2)
	{
		const size_t s = 4 * s_4, m = 4 * s;
		uint32_t root[3]; for (int k = 0; k < 3; ++k) root[k] = prroot_n(m, k);
		for (size_t i = 0; i < s_4; ++i)
		{
			for (int k = 0; k < 3; ++k)
			{
				uint32_t w[4];
				for (size_t j = 0; j < 4; ++j) w[j] = pow_p(root[k], bitrev(i + j * s_4, 2 * s) + 1, k);
				for (size_t j = 0; j < 4; ++j) wr[s_4 + i].r[k][j] = w[j];
				/* wri[s_4 + (s_4 - i - 1)] = -RNS4(w3, w2, w1, w0) */
				for (size_t j = 0; j < 4; ++j) wri[s_4 + (s_4 - i - 1)].r[k][j] = neg_p(w[3 - j], modp(k));
			}
		}
	}
	{
		const size_t s_4 = size_4 / 4, s = 4 * s_4, m = 4 * (2 * s);
		uint32_t root[3]; for (int k = 0; k < 3; ++k) root[k] = prroot_n(m, k);
		for (size_t i = 0; i < s_4; ++i)
			for (int k = 0; k < 3; ++k)
				for (size_t j = 0; j < 4; ++j) wr[2 * s_4 + i].r[k][j] = pow_p(root[k], bitrev(i + j * s_4, 2 * s) + 1, k);
	}
	/* forward0/backward0 constants (:619-633): with r16 = prRoot_n(16),
	   w1 = r16^4, w2 = r16^2, w3 = r16^6 and wi1 = -w1, wi2 = -w3, wi3 = -w2. */
	for (int k = 0; k < 3; ++k)
	{
		const uint32_t p = modp(k), r16 = prroot_n(16, k);
		t->w0[k][0] = pow_p(r16, 4, k); t->w0[k][1] = pow_p(r16, 2, k); t->w0[k][2] = pow_p(r16, 6, k);
		t->wi0[k][0] = neg_p(t->w0[k][0], p); t->wi0[k][1] = neg_p(t->w0[k][2], p); t->wi0[k][2] = neg_p(t->w0[k][1], p);
		/* Zp::norm(n) = -(p-1)/n */
		t->norm[k] = neg_p((uint32_t)((p - 1) / (t->size / 2)), p);
	}
}

/* Zp4::forward_4 / backward_4 across the 4 lanes (:172-184). */
static void lanes_forward4(rns4 *z, const uint32_t w[3][3])
{
	for (int k = 0; k < 3; ++k)
	{
		const uint32_t p = modp(k);
		const uint32_t u0 = z->r[k][0], u2 = mul_p(z->r[k][2], w[k][0], k), u1 = z->r[k][1], u3 = mul_p(z->r[k][3], w[k][0], k);
		const uint32_t v0 = add_p(u0, u2, p), v1 = mul_p(add_p(u1, u3, p), w[k][1], k);
		const uint32_t v2 = sub_p(u0, u2, p), v3 = mul_p(sub_p(u1, u3, p), w[k][2], k);
		z->r[k][0] = add_p(v0, v1, p); z->r[k][1] = sub_p(v0, v1, p);
		z->r[k][2] = add_p(v2, v3, p); z->r[k][3] = sub_p(v2, v3, p);
	}
}
static void lanes_backward4(rns4 *z, const uint32_t wi[3][3])
{
	for (int k = 0; k < 3; ++k)
	{
		const uint32_t p = modp(k);
		const uint32_t u0 = z->r[k][0], u2 = z->r[k][2], u1 = z->r[k][1], u3 = z->r[k][3];
		const uint32_t v0 = add_p(u0, u1, p), v1 = mul_p(sub_p(u0, u1, p), wi[k][1], k);
		const uint32_t v2 = add_p(u2, u3, p), v3 = mul_p(sub_p(u2, u3, p), wi[k][2], k);
		z->r[k][0] = add_p(v0, v2, p); z->r[k][1] = add_p(v1, v3, p);
		z->r[k][2] = mul_p(sub_p(v0, v2, p), wi[k][0], k); z->r[k][3] = mul_p(sub_p(v1, v3, p), wi[k][0], k);
	}
}

/* forward0 / backward0 (:619-633). */
static void forward0(const gfo_t *t, rns4 *z, size_t m) { for (size_t i = 0; i < m; ++i) lanes_forward4(&z[i], t->w0); }
static void backward0(const gfo_t *t, rns4 *z, size_t m) { for (size_t i = 0; i < m; ++i) lanes_backward4(&z[i], t->wi0); }

/* RNS4 forward_2 / forward_4 / backward_4 (:553-574). */
static void forward_2(rns4 *z, size_t k, size_t m, const rns4 *w1)
{
	rns4 *z0 = &z[k], *z1 = &z[k + m], *z2 = &z[k + 2 * m], *z3 = &z[k + 3 * m];
	const rns4 u0 = *z0, u2 = r4_mul(z2, w1), u1 = *z1, u3 = r4_mul(z3, w1);
	*z0 = r4_add(&u0, &u2); *z2 = r4_sub(&u0, &u2); *z1 = r4_add(&u1, &u3); *z3 = r4_sub(&u1, &u3);
}
static void forward_4(rns4 *z, size_t k, size_t m, const rns4 *w1, const rns4 *w2, const rns4 *w3)
{
	rns4 *z0 = &z[k], *z1 = &z[k + m], *z2 = &z[k + 2 * m], *z3 = &z[k + 3 * m];
	const rns4 u0 = *z0, u2 = r4_mul(z2, w1), u1 = *z1, u3 = r4_mul(z3, w1);
	rns4 a = r4_add(&u1, &u3), c = r4_sub(&u1, &u3);
	const rns4 v0 = r4_add(&u0, &u2), v1 = r4_mul(&a, w2), v2 = r4_sub(&u0, &u2), v3 = r4_mul(&c, w3);
	*z0 = r4_add(&v0, &v1); *z1 = r4_sub(&v0, &v1); *z2 = r4_add(&v2, &v3); *z3 = r4_sub(&v2, &v3);
}
static void backward_4(rns4 *z, size_t k, size_t m, const rns4 *wi1, const rns4 *wi2, const rns4 *wi3)
{
	rns4 *z0 = &z[k], *z1 = &z[k + m], *z2 = &z[k + 2 * m], *z3 = &z[k + 3 * m];
	const rns4 u0 = *z0, u1 = *z1, u2 = *z2, u3 = *z3;
	rns4 a = r4_sub(&u0, &u1), c = r4_sub(&u2, &u3);
	const rns4 v0 = r4_add(&u0, &u1), v1 = r4_mul(&a, wi2), v2 = r4_add(&u2, &u3), v3 = r4_mul(&c, wi3);
	rns4 d = r4_sub(&v0, &v2), e = r4_sub(&v1, &v3);
	*z0 = r4_add(&v0, &v2); *z2 = r4_mul(&d, wi1); *z1 = r4_add(&v1, &v3); *z3 = r4_mul(&e, wi1);
}

/* square_22 / square_4 / mul_22 / mul_4 (:576-617). */
static void square_22(rns4 *z, size_t k, const rns4 *w0)
{
	const rns4 u0 = z[k], u1 = z[k + 1], u2 = z[k + 2], u3 = z[k + 3];
	const rns4 t1 = r4_mul(&u1, w0), t3 = r4_mul(&u3, w0);
	rns4 a = r4_mul(&u0, &u0), b = r4_mul(&t1, &t1), c = r4_add(&u0, &u0);
	rns4 d = r4_mul(&u2, &u2), e = r4_mul(&t3, &t3), f = r4_add(&u2, &u2);
	z[k] = r4_add(&a, &b); z[k + 1] = r4_mul(&c, &u1); z[k + 2] = r4_sub(&d, &e); z[k + 3] = r4_mul(&f, &u3);
}
static void square_4(rns4 *z, size_t k, const rns4 *w0, const rns4 *w1, const rns4 *wi1)
{
	const rns4 u0 = z[k], u2 = r4_mul(&z[k + 2], w1), u1 = z[k + 1], u3 = r4_mul(&z[k + 3], w1);
	const rns4 v0 = r4_add(&u0, &u2), v2 = r4_sub(&u0, &u2), v1 = r4_add(&u1, &u3), v3 = r4_sub(&u1, &u3);
	const rns4 t1 = r4_mul(&v1, w0), t3 = r4_mul(&v3, w0);
	rns4 a = r4_mul(&v0, &v0), b = r4_mul(&t1, &t1), c = r4_add(&v0, &v0);
	rns4 d = r4_mul(&v2, &v2), e = r4_mul(&t3, &t3), f = r4_add(&v2, &v2);
	const rns4 s0 = r4_add(&a, &b), s1 = r4_mul(&c, &v1), s2 = r4_sub(&d, &e), s3 = r4_mul(&f, &v3);
	rns4 g = r4_sub(&s0, &s2), h = r4_sub(&s1, &s3);
	z[k] = r4_add(&s0, &s2); z[k + 2] = r4_mul(&g, wi1); z[k + 1] = r4_add(&s1, &s3); z[k + 3] = r4_mul(&h, wi1);
}
static void mul_22(rns4 *z, const rns4 *zp, size_t k, const rns4 *w0)
{
	const rns4 u0 = z[k], u1 = z[k + 1], u2 = z[k + 2], u3 = z[k + 3];
	const rns4 u0p = zp[k], u1p = zp[k + 1], u2p = zp[k + 2], u3p = zp[k + 3];
	const rns4 v1 = r4_mul(&u1, w0), v3 = r4_mul(&u3, w0), v1p = r4_mul(&u1p, w0), v3p = r4_mul(&u3p, w0);
	rns4 a = r4_mul(&u0, &u0p), b = r4_mul(&v1, &v1p), c = r4_mul(&u0, &u1p), d = r4_mul(&u0p, &u1);
	rns4 e = r4_mul(&u2, &u2p), f = r4_mul(&v3, &v3p), g = r4_mul(&u2, &u3p), h = r4_mul(&u2p, &u3);
	z[k] = r4_add(&a, &b); z[k + 1] = r4_add(&c, &d); z[k + 2] = r4_sub(&e, &f); z[k + 3] = r4_add(&g, &h);
}
static void mul_4(rns4 *z, const rns4 *zp, size_t k, const rns4 *w0, const rns4 *w1, const rns4 *wi1)
{
	const rns4 u0 = z[k], u2 = r4_mul(&z[k + 2], w1), u1 = z[k + 1], u3 = r4_mul(&z[k + 3], w1);
	const rns4 v0 = r4_add(&u0, &u2), v2 = r4_sub(&u0, &u2), v1 = r4_add(&u1, &u3), v3 = r4_sub(&u1, &u3);
	const rns4 v0p = zp[k], v1p = zp[k + 1], v2p = zp[k + 2], v3p = zp[k + 3];
	const rns4 t1 = r4_mul(&v1, w0), t3 = r4_mul(&v3, w0), t1p = r4_mul(&v1p, w0), t3p = r4_mul(&v3p, w0);
	rns4 a = r4_mul(&v0, &v0p), b = r4_mul(&t1, &t1p), c = r4_mul(&v0, &v1p), d = r4_mul(&v0p, &v1);
	rns4 e = r4_mul(&v2, &v2p), f = r4_mul(&t3, &t3p), g = r4_mul(&v2, &v3p), h = r4_mul(&v2p, &v3);
	const rns4 s0 = r4_add(&a, &b), s1 = r4_add(&c, &d), s2 = r4_sub(&e, &f), s3 = r4_add(&g, &h);
	rns4 x = r4_sub(&s0, &s2), y = r4_sub(&s1, &s3);
	z[k] = r4_add(&s0, &s2); z[k + 2] = r4_mul(&x, wi1); z[k + 1] = r4_add(&s1, &s3); z[k + 3] = r4_mul(&y, wi1);
}

/* forward4 / backward4 / forward2 / square22 / square4 / mul22 / mul4 (:635-670). */
static void forward4(rns4 *z, const rns4 *wr, size_t m, size_t s_4, size_t j)
{
	const rns4 *w1 = &wr[s_4 + j], *w2 = &wr[2 * (s_4 + j) + 0], *w3 = &wr[2 * (s_4 + j) + 1];
	for (size_t i = 0; i < m; ++i) forward_4(z, 4 * m * j + i, m, w1, w2, w3);
}
static void backward4(rns4 *z, const rns4 *wri, size_t m, size_t s_4, size_t j)
{
	const rns4 *wi1 = &wri[s_4 + j], *wi2 = &wri[2 * (s_4 + j) + 0], *wi3 = &wri[2 * (s_4 + j) + 1];
	for (size_t i = 0; i < m; ++i) backward_4(z, 4 * m * j + i, m, wi1, wi2, wi3);
}
static void forward2(rns4 *z, const rns4 *wr, size_t m, size_t s_4, size_t j0)
{
	for (size_t i = 0, j = j0; i < m; ++i, ++j) forward_2(z, 4 * j, 1, &wr[s_4 + j]);
}
static void square22(rns4 *z, const rns4 *wr, size_t m, size_t s_4, size_t j0)
{
	for (size_t i = 0, j = j0; i < m; ++i, ++j) square_22(z, 4 * j, &wr[2 * s_4 + j]);
}
static void square4(rns4 *z, const rns4 *wr, const rns4 *wri, size_t m, size_t s_4, size_t j0)
{
	for (size_t i = 0, j = j0; i < m; ++i, ++j) square_4(z, 4 * j, &wr[2 * s_4 + j], &wr[s_4 + j], &wri[s_4 + j]);
}
static void mul22(rns4 *z, const rns4 *zp, const rns4 *wr, size_t m, size_t s_4, size_t j0)
{
	for (size_t i = 0, j = j0; i < m; ++i, ++j) mul_22(z, zp, 4 * j, &wr[2 * s_4 + j]);
}
static void mul4(rns4 *z, const rns4 *zp, const rns4 *wr, const rns4 *wri, size_t m, size_t s_4, size_t j0)
{
	for (size_t i = 0, j = j0; i < m; ++i, ++j) mul_4(z, zp, 4 * j, &wr[2 * s_4 + j], &wr[s_4 + j], &wri[s_4 + j]);
}

/* forward / square / mul recursions (:672-741). */
static void forward_rec(rns4 *z, const rns4 *wr, size_t mr, size_t sr_4, size_t jr)
{
	if (mr >= 32)
	{
		forward4(z, wr, mr, sr_4, jr);
		for (size_t l = 0; l < 4; ++l) forward_rec(z, wr, mr / 4, 4 * sr_4, 4 * jr + l);
	}
	else
	{
		size_t m = mr;
		for (size_t s = 1; m >= 2; m /= 4, s *= 4)
			for (size_t j = 0; j < s; ++j) forward4(z, wr, m, s * sr_4, s * jr + j);
		if (m == 1) forward2(z, wr, mr, mr * sr_4, mr * jr);
	}
}
static void square_rec(rns4 *z, const rns4 *wr, const rns4 *wri, size_t mr, size_t sr_4, size_t jr)
{
	if (mr >= 32)
	{
		forward4(z, wr, mr, sr_4, jr);
		for (size_t l = 0; l < 4; ++l) square_rec(z, wr, wri, mr / 4, 4 * sr_4, 4 * jr + l);
		backward4(z, wri, mr, sr_4, jr);
	}
	else
	{
		size_t m = mr;
		for (size_t s = 1; m >= 2; m /= 4, s *= 4)
			for (size_t j = 0; j < s; ++j) forward4(z, wr, m, s * sr_4, s * jr + j);
		if (m == 0) square22(z, wr, mr, mr * sr_4, mr * jr); else square4(z, wr, wri, mr, mr * sr_4, mr * jr);
		m = (m == 0) ? 2 : 4;
		for (size_t s = mr / m; m <= mr; m *= 4, s /= 4)
			for (size_t j = 0; j < s; ++j) backward4(z, wri, m, s * sr_4, s * jr + j);
	}
}
static void mul_rec(rns4 *z, const rns4 *zp, const rns4 *wr, const rns4 *wri, size_t mr, size_t sr_4, size_t jr)
{
	if (mr >= 32)
	{
		forward4(z, wr, mr, sr_4, jr);
		for (size_t l = 0; l < 4; ++l) mul_rec(z, zp, wr, wri, mr / 4, 4 * sr_4, 4 * jr + l);
		backward4(z, wri, mr, sr_4, jr);
	}
	else
	{
		size_t m = mr;
		for (size_t s = 1; m >= 2; m /= 4, s *= 4)
			for (size_t j = 0; j < s; ++j) forward4(z, wr, m, s * sr_4, s * jr + j);
		if (m == 0) mul22(z, zp, wr, mr, mr * sr_4, mr * jr); else mul4(z, zp, wr, wri, mr, mr * sr_4, mr * jr);
		m = (m == 0) ? 2 : 4;
		for (size_t s = mr / m; m <= mr; m *= 4, s /= 4)
			for (size_t j = 0; j < s; ++j) backward4(z, wri, m, s * sr_4, s * jr + j);
	}
}

/* garner3 (:482-503): CRT of the three residues, centred in (-M/2, M/2]. */
static i128 garner3(uint32_t r1, uint32_t r2, uint32_t r3)
{
	static uint32_t invP2_P1 = 0, invP3_P1 = 0, invP3_P2 = 0;
	if (invP2_P1 == 0)
	{
		invP2_P1 = pow_p(P2 % P1, P1 - 2, 0);
		invP3_P1 = pow_p(P3 % P1, P1 - 2, 0);
		invP3_P2 = pow_p(P3 % P2, P2 - 2, 1);
	}
	const u128 M = (u128)P1 * P2 * P3, M_2 = M >> 1;
	const uint32_t u13 = mul1(sub_p(r1, r3 % P1, P1), invP3_P1);
	const uint32_t u23 = mul2(sub_p(r2, r3 % P2, P2), invP3_P2);
	const uint32_t u123 = mul1(sub_p(u13, u23 % P1, P1), invP2_P1);
	const u128 v = (u128)u123 * ((uint64_t)P2 * P3) + (u128)u23 * P3 + r3;
	return (v > M_2) ? (i128)v - (i128)M : (i128)v;
}

/* reduce96 / reduce64 (:445-480): digit = f rem b (sign of f), f <- f quo b. */
static inline int32_t reduce(i128 *f, uint32_t b)
{
	const i128 q = *f / (i128)b, r = *f - q * (i128)b;
	*f = q;
	return (int32_t)r;
}

static inline void set_digit(rns4 *z, int lane, int32_t d)
{
	z->r[0][lane] = from_int(d, P1); z->r[1][lane] = from_int(d, P2); z->r[2][lane] = from_int(d, P3);
}

/* baseMod (:743-772). */
static void baseMod(gfo_t *t, rns4 *z, int dup)
{
	const size_t n = t->size_4;
	const uint32_t b = t->b;
	i128 f[4] = { 0, 0, 0, 0 };
	for (size_t k = 0; k < n; ++k)
	{
		rns4 x;
		for (int p = 0; p < 3; ++p) for (int l = 0; l < 4; ++l) x.r[p][l] = mul_p(z[k].r[p][l], t->norm[p], p);
		for (int l = 0; l < 4; ++l)
		{
			i128 v = garner3(x.r[0][l], x.r[1][l], x.r[2][l]);
			if (dup) v += v;
			f[l] += v;
			set_digit(&z[k], l, reduce(&f[l], b));
		}
	}
	/* int96 -> int64 carries (f96.get64()) */
	int64_t c[4]; for (int l = 0; l < 4; ++l) c[l] = (int64_t)f[l];
	while ((c[0] | c[1] | c[2] | c[3]) != 0)
	{
		/* int64_4::rotate: a_0 = -a_n (:273) */
		const int64_t c3 = c[3]; c[3] = c[2]; c[2] = c[1]; c[1] = c[0]; c[0] = -c3;
		for (size_t k = 0; k < n; ++k)
		{
			for (int l = 0; l < 4; ++l)
			{
				i128 g = (i128)c[l] + to_int(z[k].r[0][l], P1);
				set_digit(&z[k], l, reduce(&g, b));
				c[l] = (int64_t)g;
			}
			if ((c[0] | c[1] | c[2] | c[3]) == 0) return;
		}
	}
}

/* baseModMul (src/transformCPUi32.h:774-797): digits times a, then carry. */
static void baseModMul(gfo_t *t, rns4 *z, int32_t a)
{
	const size_t n = t->size_4;
	const uint32_t b = t->b;
	i128 f[4] = { 0, 0, 0, 0 };
	for (size_t k = 0; k < n; ++k)
		for (int l = 0; l < 4; ++l)
		{
			f[l] += (i128)to_int(z[k].r[0][l], P1) * a;
			set_digit(&z[k], l, reduce(&f[l], b));
		}
	int64_t c[4]; for (int l = 0; l < 4; ++l) c[l] = (int64_t)f[l];
	while ((c[0] | c[1] | c[2] | c[3]) != 0)
	{
		const int64_t c3 = c[3]; c[3] = c[2]; c[2] = c[1]; c[1] = c[0]; c[0] = -c3;
		for (size_t k = 0; k < n; ++k)
		{
			for (int l = 0; l < 4; ++l)
			{
				i128 g = (i128)c[l] + to_int(z[k].r[0][l], P1);
				set_digit(&z[k], l, reduce(&g, b));
				c[l] = (int64_t)g;
			}
			if ((c[0] | c[1] | c[2] | c[3]) == 0) return;
		}
	}
}

/* ---------------- public C ABI (checker only) ---------------- */

GFO_API void *gfo_create(uint32_t b, uint32_t n, size_t num_regs)
{
	if ((n < 5) || (n > 24) || (b < 2) || (num_regs < 1)) return NULL;
	gfo_t *t = (gfo_t *)calloc(1, sizeof(gfo_t));
	if (t == NULL) return NULL;
	t->b = b; t->n = n; t->size = (size_t)1 << n; t->size_4 = t->size / 4; t->num_regs = num_regs;
	t->z = (rns4 *)calloc(t->size_4 * num_regs, sizeof(rns4));
	t->wr = (rns4 *)calloc(2 * t->size_4, sizeof(rns4));
	t->zp = (rns4 *)calloc(t->size_4, sizeof(rns4));
	if ((t->z == NULL) || (t->wr == NULL) || (t->zp == NULL)) { free(t->z); free(t->wr); free(t->zp); free(t); return NULL; }
	build_roots(t);
	return t;
}

GFO_API void gfo_destroy(void *h)
{
	gfo_t *t = (gfo_t *)h;
	if (t == NULL) return;
	free(t->z); free(t->wr); free(t->zp); free(t);
}

/* set (:848-855) */
GFO_API void gfo_set(void *h, uint32_t a)
{
	gfo_t *t = (gfo_t *)h;
	memset(t->z, 0, t->size_4 * sizeof(rns4));
	t->z[0].r[0][0] = a % P1; t->z[0].r[1][0] = a % P2; t->z[0].r[2][0] = a % P3;
}

/* squareDup (:857-868) */
GFO_API void gfo_square_dup(void *h, int dup)
{
	gfo_t *t = (gfo_t *)h;
	const size_t size_4 = t->size_4;
	forward0(t, t->z, size_4);
	square_rec(t->z, t->wr, &t->wr[size_4], size_4 / 4, 1, 0);
	backward0(t, t->z, size_4);
	baseMod(t, t->z, dup);
}

/* squareMul (:870-874) */
GFO_API void gfo_square_mul(void *h, int32_t a)
{
	gfo_t *t = (gfo_t *)h;
	gfo_square_dup(h, 0);
	baseModMul(t, t->z, a);
}

/* initMultiplicand (:876-886) */
GFO_API void gfo_init_multiplicand(void *h, size_t src)
{
	gfo_t *t = (gfo_t *)h;
	const size_t size_4 = t->size_4;
	memcpy(t->zp, &t->z[src * size_4], size_4 * sizeof(rns4));
	forward0(t, t->zp, size_4);
	forward_rec(t->zp, t->wr, size_4 / 4, 1, 0);
}

/* mul (:888-899) */
GFO_API void gfo_mul(void *h)
{
	gfo_t *t = (gfo_t *)h;
	const size_t size_4 = t->size_4;
	forward0(t, t->z, size_4);
	mul_rec(t->z, t->zp, t->wr, &t->wr[size_4], size_4 / 4, 1, 0);
	backward0(t, t->z, size_4);
	baseMod(t, t->z, 0);
}

/* copy (:901-907) */
GFO_API void gfo_copy(void *h, size_t dst, size_t src)
{
	gfo_t *t = (gfo_t *)h;
	if (dst == src) return;
	memcpy(&t->z[dst * t->size_4], &t->z[src * t->size_4], t->size_4 * sizeof(rns4));
}

/* getZi (:800-810): digit i = lane i/(N/4), element i%(N/4), signed from prime 1. */
GFO_API void gfo_get_zi(const void *h, int32_t *zi)
{
	const gfo_t *t = (const gfo_t *)h;
	const size_t size_4 = t->size_4;
	for (size_t k = 0; k < size_4; ++k)
		for (int l = 0; l < 4; ++l) zi[l * size_4 + k] = to_int(t->z[k].r[0][l], P1);
}

/* setZi (:812-825) */
GFO_API void gfo_set_zi(void *h, const int32_t *zi)
{
	gfo_t *t = (gfo_t *)h;
	const size_t size_4 = t->size_4;
	for (size_t k = 0; k < size_4; ++k)
		for (int l = 0; l < 4; ++l) set_digit(&t->z[k], l, zi[l * size_4 + k]);
}

/* Raw register 0 state (3 primes x 4 lanes per element), for bit-level
   comparison against the reference's saveContext payload (:839-846). */
GFO_API void gfo_get_raw(const void *h, uint32_t *out)
{
	const gfo_t *t = (const gfo_t *)h;
	memcpy(out, t->z, t->size_4 * sizeof(rns4));
}

/* ---------------- gint restatement (src/gint.h) ---------------- */

/* gint::unbalance (src/gint.h:40-102, non-CYCLO branch). */
GFO_API void gfo_unbalance(int32_t *d, size_t size, uint32_t base_u)
{
	const int32_t base = (int32_t)base_u;
	int64_t f = 0;
	for (size_t i = 0; i < size; ++i)
	{
		f += d[i];
		int32_t r = (int32_t)(f % base);
		if (r < 0) r += base;
		d[i] = r; f -= r; f /= base;
	}
	while (f != 0)
	{
		f = -f;
		for (size_t i = 0; i < size; ++i)
		{
			f += d[i];
			int32_t r = (int32_t)(f % base);
			if (r < 0) r += base;
			d[i] = r; f -= r; f /= base;
			if (f == 0) break;
		}
		if (f == 1)
		{
			int isMinusOne = 1;
			for (size_t i = 0; i < size; ++i) if (d[i] != 0) { isMinusOne = 0; break; }
			if (isMinusOne) { d[0] = -1; break; }
		}
	}
}

/* gint::balance (src/gint.h:104-149, non-CYCLO branch). */
GFO_API void gfo_balance(int32_t *d, size_t size, uint32_t base_u)
{
	const int32_t base = (int32_t)base_u;
	int64_t f = 0;
	for (size_t i = 0; i < size; ++i)
	{
		f += d[i];
		int32_t r = (int32_t)(f % base);
		if (r > base / 2) r -= base;
		if (r <= -base / 2) r += base;
		d[i] = r; f -= r; f /= base;
	}
	while (f != 0)
	{
		f = -f;
		for (size_t i = 0; i < size; ++i)
		{
			f += d[i];
			int32_t r = (int32_t)(f % base);
			if (r > base / 2) r -= base;
			if (r <= -base / 2) r += base;
			d[i] = r; f -= r; f /= base;
			if (f == 0) break;
		}
	}
}

/* gint::isOne on unbalanced digits (src/gint.h:169-202, non-CYCLO): returns
   isOne, writes res64 and old64. */
GFO_API int gfo_is_one(const int32_t *d, size_t size, uint32_t base, uint64_t *res64, uint64_t *old64)
{
	int bOne = (d[0] == 1);
	if (bOne) for (size_t i = 1; i < size; ++i) bOne &= (d[i] == 0);
	uint64_t r64 = 0, bb = 1;
	for (size_t i = 0; i < size; ++i) { r64 += (uint64_t)(uint32_t)d[i] * bb; bb *= base; }
	*res64 = r64;
	uint64_t old = 0;
	for (size_t i = 8; i != 0; --i) old = (old << 8) | (uint8_t)d[size - i];
	*old64 = old;
	return bOne;
}

static inline uint64_t rotl64(uint64_t x, uint8_t n) { return (x << n) | (x >> (-n & 63)); }

/* gint::gethash64 on unbalanced digits (src/gint.h:204-219). */
GFO_API uint64_t gfo_hash64(const int32_t *d, size_t size)
{
	uint64_t hash = 0;
	for (size_t i = 0; i < size; ++i)
	{
		const uint32_t a_i = (uint32_t)d[i];
		hash += a_i;
		hash ^= rotl64(a_i + 0xc39d8a0552b073e8ull, (uint8_t)((17 * (uint64_t)a_i + 5) % 64));
	}
	return hash;
}
