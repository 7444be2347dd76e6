// gf_arith.cuh -- exact modular and multi-word integer arithmetic for the
// B200 modular-squaring engine (integer pipe only; no floating point).
//
// Two RNS prime sets (one is chosen per test from b and n):
//   set 0: W = 2 primes just below 2^32  (widest exact range for two planes)
//   set 1: W = 3 primes just below 2^31  (every 12 <= n <= 23, b < 2^31;
//          31-bit primes let add/sub/Montgomery use min() corrections)
// The primes are the NTT-friendly primes genefer's transforms use
// (src/transformCPUi32.h:19-21 and src/transformGPU.h:37-105: 125*2^25+1,
// 243*2^24+1; 127*2^24+1, 63*2^25+1, 15*2^27+1).  Products of two residues
// are Montgomery products with R = 2^32 (Montgomery 1985); products by a root
// of the transform tables are Montgomery products for the 32-bit primes and
// Shoup products (a precomputed quotient per root, Shoup 2007) for the 31-bit
// primes; residues are always fully reduced to [0, p).
#pragma once

#include <cstdint>
#include <type_traits>

namespace gfc {

typedef unsigned __int128 u128;
typedef __int128 i128;

// ---------------------------------------------------------------- constexpr helpers

__host__ __device__ constexpr uint32_t mont_qinv(uint32_t p)
{
	// p^{-1} mod 2^32 by Newton iteration (x <- x (2 - p x)).
	uint32_t x = p;
	for (int i = 0; i < 5; ++i) x *= 2u - p * x;
	return x;
}

__host__ __device__ constexpr uint32_t powmod_c(uint32_t a, uint64_t e, uint32_t p)
{
	uint64_t r = 1, y = a % p;
	while (e != 0) { if (e & 1) r = (r * y) % p; y = (y * y) % p; e >>= 1; }
	return static_cast<uint32_t>(r);
}

__host__ __device__ constexpr uint32_t invmod_c(uint32_t a, uint32_t p) { return powmod_c(a, p - 2, p); }

// x * 2^32 mod p  (Montgomery form of x)
__host__ __device__ constexpr uint32_t to_mont_c(uint32_t x, uint32_t p)
{
	return static_cast<uint32_t>((static_cast<uint64_t>(x % p) << 32) % p);
}

// ---------------------------------------------------------------- prime sets

template <int SET> struct PrimeSet;

template <> struct PrimeSet<0>
{
	static constexpr int W = 2;
	static constexpr bool P31 = false;
	static constexpr uint32_t p[4] = { 125u * (1u << 25) + 1u, 243u * (1u << 24) + 1u, 0u, 0u };
};

template <> struct PrimeSet<1>
{
	static constexpr int W = 3;
	static constexpr bool P31 = true;
	static constexpr uint32_t p[4] = { 127u * (1u << 24) + 1u, 63u * (1u << 25) + 1u, 15u * (1u << 27) + 1u, 0u };
};

// Set 2: four primes below 2^31 for packed digits (two base-b digits per
// coefficient of a transform of N/2 points); the fourth, 249 * 2^23 + 1, has
// 2^23 | p - 1, enough for N/2 <= 2^22.
template <> struct PrimeSet<2>
{
	static constexpr int W = 4;
	static constexpr bool P31 = true;
	static constexpr uint32_t p[4] = { 127u * (1u << 24) + 1u, 63u * (1u << 25) + 1u, 249u * (1u << 23) + 1u,
									   15u * (1u << 27) + 1u };
};

// ---------------------------------------------------------------- Zp (one prime)

// A root of the transform tables as its prime's product by it wants it: one
// word in Montgomery form for the 32-bit primes; for the 31-bit primes the
// root w in normal form with its Shoup quotient q = floor(w 2^32 / p).
struct RootM { uint32_t w; };
struct RootS { uint32_t w, q; };

// w and floor(w 2^32 / p), at compile time
__host__ __device__ constexpr RootS shoup_c(uint32_t w, uint32_t p)
{
	return RootS{ w, static_cast<uint32_t>((static_cast<uint64_t>(w) << 32) / p) };
}

// a w mod p for a < 2^32, w < p < 2^31 (Shoup): with h = floor(a q / 2^32),
// a w - h p lies in [0, 2p), so its low 32 bits are exact.
__device__ __forceinline__ uint32_t shoup_mul(uint32_t a, RootS r, uint32_t p)
{
	const uint32_t h = __umulhi(a, r.q);
	const uint32_t t = a * r.w - h * p;
	return min(t, t - p);
}

template <uint32_t P, bool P31>
struct Zp
{
	static constexpr uint32_t p = P;
	static constexpr uint32_t q = mont_qinv(P);   // p * q = 1 (mod 2^32)

	__device__ __forceinline__ static uint32_t add(uint32_t a, uint32_t b)
	{
		const uint32_t s = a + b;
		if (P31) return min(s, s - P);
		return (a >= P - b) ? s - P : s;
	}

	__device__ __forceinline__ static uint32_t sub(uint32_t a, uint32_t b)
	{
		const uint32_t d = a - b;
		if (P31) return min(d, d + P);
		return (a < b) ? d + P : d;
	}

	// a * b * 2^-32 mod p, for a < 2^32 and b < p (result in [0, p)).
	__device__ __forceinline__ static uint32_t mul(uint32_t a, uint32_t b)
	{
		const uint64_t t = static_cast<uint64_t>(a) * b;
		const uint32_t lo = static_cast<uint32_t>(t), hi = static_cast<uint32_t>(t >> 32);
		const uint32_t mh = __umulhi(lo * q, P);
		const uint32_t u = hi - mh;
		if (P31) return min(u, u + P);
		return (hi < mh) ? u + P : u;
	}

	// t 2^-32 mod p for t < p 2^32 (Montgomery reduction; result in [0, p)).
	__device__ __forceinline__ static uint32_t redc64(uint64_t t)
	{
		const uint32_t lo = static_cast<uint32_t>(t), hi = static_cast<uint32_t>(t >> 32);
		const uint32_t mh = __umulhi(lo * q, P);
		const uint32_t u = hi - mh;
		if (P31) return min(u, u + P);
		return (hi < mh) ? u + P : u;
	}

	// signed digit -> residue (|d| < p)
	__device__ __forceinline__ static uint32_t from_int(int32_t d)
	{
		return static_cast<uint32_t>(d) + ((d < 0) ? P : 0u);
	}

	// a times a table root (a w mod p)
	using root_t = typename std::conditional<P31, RootS, RootM>::type;
	__device__ __forceinline__ static uint32_t mulr(uint32_t a, RootS r) { return shoup_mul(a, r, P); }
	__device__ __forceinline__ static uint32_t mulr(uint32_t a, RootM r) { return mul(a, r.w); }
};

// The same arithmetic with the prime held in registers, so that one code path
// serves every plane of a prime set (smaller kernels, fewer i-cache misses).
template <bool P31>
struct ZpR
{
	uint32_t p, q;

	__device__ __forceinline__ uint32_t add(uint32_t a, uint32_t b) const
	{
		const uint32_t s = a + b;
		if (P31) return min(s, s - p);
		return (a >= p - b) ? s - p : s;
	}

	__device__ __forceinline__ uint32_t sub(uint32_t a, uint32_t b) const
	{
		const uint32_t d = a - b;
		if (P31) return min(d, d + p);
		return (a < b) ? d + p : d;
	}

	__device__ __forceinline__ uint32_t mul(uint32_t a, uint32_t b) const
	{
		const uint64_t t = static_cast<uint64_t>(a) * b;
		const uint32_t lo = static_cast<uint32_t>(t), hi = static_cast<uint32_t>(t >> 32);
		const uint32_t mh = __umulhi(lo * q, p);
		const uint32_t u = hi - mh;
		if (P31) return min(u, u + p);
		return (hi < mh) ? u + p : u;
	}

	__device__ __forceinline__ uint32_t redc64(uint64_t t) const
	{
		const uint32_t lo = static_cast<uint32_t>(t), hi = static_cast<uint32_t>(t >> 32);
		const uint32_t mh = __umulhi(lo * q, p);
		const uint32_t u = hi - mh;
		if (P31) return min(u, u + p);
		return (hi < mh) ? u + p : u;
	}

	__device__ __forceinline__ uint32_t from_int(int32_t d) const
	{
		return static_cast<uint32_t>(d) + ((d < 0) ? p : 0u);
	}

	using root_t = typename std::conditional<P31, RootS, RootM>::type;
	__device__ __forceinline__ uint32_t mulr(uint32_t a, RootS r) const { return shoup_mul(a, r, p); }
	__device__ __forceinline__ uint32_t mulr(uint32_t a, RootM r) const { return mul(a, r.w); }
};

// Plane `pl` of prime set SET as register-held arithmetic.
template <int SET>
__device__ __forceinline__ ZpR<PrimeSet<SET>::P31> prime_rt(int pl)
{
	constexpr uint32_t p0 = PrimeSet<SET>::p[0], p1 = PrimeSet<SET>::p[1], p2 = PrimeSet<SET>::p[2],
					   p3 = PrimeSet<SET>::p[3];
	ZpR<PrimeSet<SET>::P31> z;
	z.p = (pl == 0) ? p0 : ((pl == 1) ? p1 : ((pl == 2) ? p2 : p3));
	z.q = (pl == 0) ? mont_qinv(p0) : ((pl == 1) ? mont_qinv(p1) : ((pl == 2) ? mont_qinv(p2) : mont_qinv(p3)));
	return z;
}

// ---------------------------------------------------------------- CRT (Garner)

// Host-side constants, computed once per prime set.
template <int SET>
struct Crt;

template <>
struct Crt<0>
{
	// v = x1 + p1 * a2,  a2 = (x2 - x1) * p1^{-1} mod p2
	static constexpr uint32_t p1 = PrimeSet<0>::p[0], p2 = PrimeSet<0>::p[1];
	static constexpr uint32_t c12 = to_mont_c(invmod_c(p1 % p2, p2), p2);   // p1^{-1} in Montgomery form mod p2
};

template <>
struct Crt<1>
{
	// Garner's constants with their Shoup quotients (the set-1 primes are below 2^31):
	// p1^-1 mod p2, p1 mod p3, (p1 p2)^-1 mod p3
	static constexpr uint32_t p1 = PrimeSet<1>::p[0], p2 = PrimeSet<1>::p[1], p3 = PrimeSet<1>::p[2];
	static constexpr RootS s12 = shoup_c(invmod_c(p1 % p2, p2), p2);
	static constexpr RootS s1_3 = shoup_c(p1 % p3, p3);
	static constexpr RootS s123 = shoup_c(invmod_c(static_cast<uint32_t>((static_cast<uint64_t>(p1) * p2) % p3), p3), p3);
};

template <>
struct Crt<2>
{
	// as Crt<1>, and p1 mod p4, p1 p2 mod p4, (p1 p2 p3)^-1 mod p4 (every set-2 prime is below 2^31)
	static constexpr uint32_t p1 = PrimeSet<2>::p[0], p2 = PrimeSet<2>::p[1], p3 = PrimeSet<2>::p[2], p4 = PrimeSet<2>::p[3];
	static constexpr RootS s12 = shoup_c(invmod_c(p1 % p2, p2), p2);
	static constexpr RootS s1_3 = shoup_c(p1 % p3, p3);
	static constexpr RootS s123 = shoup_c(invmod_c(static_cast<uint32_t>((static_cast<uint64_t>(p1) * p2) % p3), p3), p3);
	static constexpr RootS s1_4 = shoup_c(p1 % p4, p4);
	static constexpr RootS s12_4 = shoup_c(static_cast<uint32_t>((static_cast<uint64_t>(p1) * p2) % p4), p4);
	static constexpr RootS s1234 = shoup_c(invmod_c(static_cast<uint32_t>(
		(((static_cast<uint64_t>(p1) * p2) % p4) * p3) % p4), p4), p4);
};

// ---------------------------------------------------------------- CRT + base-b carry

// Division by a fixed base b (2 <= b < 2^31) with the 64-bit reciprocal
// binv = floor((2^64 - 1) / b): for n < 2^64, q = mulhi(n, binv) is floor(n/b)
// or one less (Barrett 1986), fixed by one compare.
__device__ __forceinline__ uint64_t divb64(uint64_t n, uint32_t b, uint64_t binv, uint64_t &r)
{
	uint64_t q = __umul64hi(n, binv);
	uint64_t rr = n - q * b;
	if (rr >= b) { q += 1; rr -= b; }
	r = rr;
	return q;
}

// Per-test constants of the fused CRT + carry, computed on the host.
// With f = 1 (square) or 2 (dup), T the top mixed-radix weight of the prime
// set (p1 for set 0, p1 p2 for set 1) and M the product of its primes:
//   q[f-1] = floor(f T / b), r[f-1] = f T mod b,
//   mq[f-1] = floor(f M / b) mod 2^64, mr[f-1] = f M mod b,
//   K = ceil(2^56 / b), kb = K b;  K' = ceil(2^62 / b), kwb = K' b.
struct CarryK
{
	uint64_t binv, kb, k;
	uint64_t kw, kwb;       // K' = ceil(2^62 / b), K' b: the same for |s| < 2^62
	uint64_t q[2], mq[2];
	uint32_t r[2], mr[2];
	uint32_t b, h;
};

// Balanced digit in [-b/2, b/2) of f v + c, where v is the centred CRT value
// of the residues x (|v| < M/2), and the carry floor((f v + c + b/2) / b)
// written back to c.  Garner's mixed radix v = x1 + p1 a2 (+ p1 p2 a3) is
// split as  f v + c + b/2 = U + c + b (Q top - z (mq + 1))  with the top term
// f T top = (Q b + R) top folded into U < 2^64, so one 64-bit division by b
// remains; the quotient is assembled modulo 2^64, which is exact because the
// carry of a resting register is below 2^55 in magnitude.
//
// crt_split does everything that does not depend on c: u = U + K b and
// t = Q top - z (mq + 1) - K (both modulo 2^64); crt_chain then adds the
// carry, divides once and returns the digit.  crt_carry is the two in one.
template <int SET>
__device__ __forceinline__ void crt_split(const uint32_t x[3], int dup, const CarryK &K, uint64_t &u, uint64_t &t);

template <>
__device__ __forceinline__ void crt_split<0>(const uint32_t x[3], int dup, const CarryK &K, uint64_t &u, uint64_t &t)
{
	using C = Crt<0>;
	using Z2 = Zp<C::p2, false>;
	constexpr uint64_t M = static_cast<uint64_t>(C::p1) * C::p2;
	const uint32_t x1m2 = (x[0] >= C::p2) ? x[0] - C::p2 : x[0];
	const uint32_t a2 = Z2::mul(Z2::sub(x[1], x1m2), C::c12);
	const bool z = (static_cast<uint64_t>(a2) * C::p1 + x[0]) > M / 2;
	u = (static_cast<uint64_t>(x[0]) << dup) + static_cast<uint64_t>(K.r[dup]) * a2 + K.h + (z ? K.b - K.mr[dup] : 0u) + K.kb;
	t = K.q[dup] * a2 - (z ? K.mq[dup] + 1 : 0) - K.k;
}

template <>
__device__ __forceinline__ void crt_split<1>(const uint32_t x[3], int dup, const CarryK &K, uint64_t &u, uint64_t &t)
{
	using C = Crt<1>;
	using Z2 = Zp<C::p2, true>;
	using Z3 = Zp<C::p3, true>;
	constexpr uint64_t P12 = static_cast<uint64_t>(C::p1) * C::p2;
	const uint32_t x1m2 = (x[0] >= C::p2) ? x[0] - C::p2 : x[0];
	const uint32_t a2 = shoup_mul(Z2::sub(x[1], x1m2), C::s12, C::p2);
	const uint32_t x1m3 = (x[0] >= C::p3) ? x[0] - C::p3 : x[0];
	const uint32_t a3 = shoup_mul(Z3::sub(x[2], Z3::add(x1m3, shoup_mul(a2, C::s1_3, C::p3))), C::s123, C::p3);
	const uint64_t low = static_cast<uint64_t>(a2) * C::p1 + x[0];          // < p1 p2
	const bool z = (a3 > (C::p3 - 1) / 2) || ((a3 == (C::p3 - 1) / 2) && (low > P12 / 2));
	u = (low << dup) + static_cast<uint64_t>(K.r[dup]) * a3 + K.h + (z ? K.b - K.mr[dup] : 0u) + K.kb;
	t = K.q[dup] * a3 - (z ? K.mq[dup] + 1 : 0) - K.k;
}

__device__ __forceinline__ int32_t crt_chain(uint64_t u, uint64_t t, const CarryK &K, int64_t &c)
{
	uint64_t rv;
	const uint64_t qv = divb64(u + static_cast<uint64_t>(c), K.b, K.binv, rv);
	c = static_cast<int64_t>(qv + t);
	return static_cast<int32_t>(rv) - static_cast<int32_t>(K.h);
}

template <int SET>
__device__ __forceinline__ int32_t crt_carry(const uint32_t x[3], int dup, const CarryK &K, int64_t &c)
{
	uint64_t u, t;
	crt_split<SET>(x, dup, K, u, t);
	return crt_chain(u, t, K, c);
}

// Balanced digit of s (|s| < 2^62) and carry floor((s + b/2) / b).
__device__ __forceinline__ int32_t carry_wide(int64_t s, const CarryK &K, int64_t &c)
{
	uint64_t rv;
	const uint64_t qv = divb64(static_cast<uint64_t>(s) + K.h + K.kwb, K.b, K.binv, rv);
	c = static_cast<int64_t>(qv - K.kw);
	return static_cast<int32_t>(rv) - static_cast<int32_t>(K.h);
}

// Balanced digit of s (|s| < 2^56) and carry floor((s + b/2) / b).
__device__ __forceinline__ int32_t carry_small(int64_t s, const CarryK &K, int64_t &c)
{
	uint64_t rv;
	const uint64_t qv = divb64(static_cast<uint64_t>(s) + K.h + K.kb, K.b, K.binv, rv);
	c = static_cast<int64_t>(qv - K.k);
	return static_cast<int32_t>(rv) - static_cast<int32_t>(K.h);
}

// ---------------------------------------------------------------- packed digits (set 2)
//
// A coefficient of the packed transform is D = d0 + b d1 for two consecutive
// balanced base-b digits.  After the inverse transform its CRT value is f V
// (f = 1, or 2 for a doubled square), |V| < M/2 with M = p1 p2 p3 p4 < 2^124.
// Garner gives V = a1 + p1 a2 + p1 p2 a3 + p1 p2 p3 a4' with a_k < p_k and
// a4' = a4, or a4 - p4 when the value a1 + ... + p1 p2 p3 a4 exceeds M/2 (then
// it is V + M, and M = p1 p2 p3 p4).  Every weight w = f p1 ... p_{k-1} is
// written in base b on the host (limbs < b < 2^28), so that
//     f V = sum_{j<5} U_j b^j,   U_j = sum_k a_k w_{k,j},
// a sum of products of (signed) 31- and 28-bit numbers.  The limbs shrink
// with j (w1 < 2^33, w2 < 2^64, w3 < 2^95 and b >= 2^20 give |U_0|, |U_1| <
// 2^60.6, |U_2| < 2^60, |U_3| < 2^59.1, |U_4| < 2^45), and a window position p
// collects U_{p-2i} of at most three coefficients i plus the carry of the
// digit before it, so every position stays below 2^61.4 in magnitude: the U_j
// are added to the window unsplit, two digits are completed per coefficient
// (one 64-bit division each), and what remains after a 16-digit segment
// (positions 16 .. 20) is the segment's carry, five values below 2^62 added to
// the next segment's first five digits.

constexpr int PK_CARRY = 5;     // carry values per 16-digit segment

// Per-test constants of the packed CRT + carry (host-computed); index f - 1.
struct PackK
{
	uint32_t w1[2][2];          // limbs 0..1 of f p1
	uint32_t w2[2][4];          // limbs 0..3 of f p1 p2
	uint32_t w3[2][5];          // limbs 0..4 of f p1 p2 p3
	uint32_t bm[4];             // b mod p_k in Montgomery form (packing d0 + b d1 in 16-row columns)
};

// A packed coefficient D = d0 + b d1 of two resting digits (|d| <= b/2 + 1,
// b < 2^28: |D| < 2^55) as the residue D 2^-32 mod p of a set-2 prime: one
// Montgomery reduction of D + 2^25 p, which lies in (0, p 2^32) since
// p > 2^30.  The 8-row packed column kernels pack this way; the factor 2^-32
// on their inputs is compensated by the normalisation in word 1 of entry 0
// of the set-2 root tables (word 0 holds the one for D itself, which the
// 16-row column kernels make as d0 + (b mod p) d1).
__device__ __forceinline__ int64_t pack_value(int32_t d0, int32_t d1, uint32_t b)
{
	return static_cast<int64_t>(d0) + static_cast<int64_t>(static_cast<int32_t>(b)) * static_cast<int64_t>(d1);
}

template <class Z>
__device__ __forceinline__ uint32_t pack_residue(const Z &z, int64_t D)
{
	return z.redc64(static_cast<uint64_t>(D + (static_cast<int64_t>(z.p) << 25)));
}

// Garner's mixed-radix digits a1..a4 of one packed coefficient (residues
// x[4]), a4 carrying in bit 31 the flag V > M/2 (a4 < p4 < 2^31).
__device__ __forceinline__ void crt_garner4(uint32_t (&x)[4])
{
	using C = Crt<2>;
	using Z2 = Zp<C::p2, true>;
	using Z3 = Zp<C::p3, true>;
	using Z4 = Zp<C::p4, true>;
	const uint32_t a1 = x[0];
	const uint32_t a1m2 = (a1 >= C::p2) ? a1 - C::p2 : a1;
	const uint32_t a2 = shoup_mul(Z2::sub(x[1], a1m2), C::s12, C::p2);
	const uint32_t a1m3 = (a1 >= C::p3) ? a1 - C::p3 : a1;
	const uint32_t a3 = shoup_mul(Z3::sub(x[2], Z3::add(a1m3, shoup_mul(a2, C::s1_3, C::p3))), C::s123, C::p3);
	const uint32_t a1m4 = (a1 >= C::p4) ? a1 - C::p4 : a1;
	const uint32_t s4 = Z4::add(Z4::add(a1m4, shoup_mul(a2, C::s1_4, C::p4)), shoup_mul(a3, C::s12_4, C::p4));
	const uint32_t a4 = shoup_mul(Z4::sub(x[3], s4), C::s1234, C::p4);
	// V > M/2 by mixed-radix digits from the top (M/2 = T (p4 - 1)/2 + T/2, T = p1 p2 p3)
	constexpr uint64_t P12 = static_cast<uint64_t>(C::p1) * C::p2;
	const uint64_t low = static_cast<uint64_t>(a2) * C::p1 + a1;            // < p1 p2
	const bool rest_hi = (a3 > (C::p3 - 1) / 2) || ((a3 == (C::p3 - 1) / 2) && (low > P12 / 2));
	const bool z = (a4 > (C::p4 - 1) / 2) || ((a4 == (C::p4 - 1) / 2) && rest_hi);
	x[0] = a1; x[1] = a2; x[2] = a3; x[3] = a4 | (z ? 0x80000000u : 0u);
}

// Adds f V (mixed-radix digits g from crt_garner4) to the window at
// positions 0..4.
__device__ __forceinline__ void crt_window_g(const uint32_t (&g)[4], int dup, const PackK &P, int64_t (&win)[7])
{
	const int f = dup;                                                       // index f - 1
	const uint64_t A1 = g[0], A2 = g[1], A3 = g[2];
	// the top digit, less p4 for the centred value V > M/2 (M = p1 p2 p3 p4)
	const int64_t A4 = static_cast<int64_t>(g[3] & 0x7fffffffu) - ((g[3] >> 31) ? static_cast<int64_t>(Crt<2>::p4) : 0);
	win[0] += static_cast<int64_t>((A1 << dup) + A2 * P.w1[f][0] + A3 * P.w2[f][0]) + A4 * static_cast<int64_t>(P.w3[f][0]);
	win[1] += static_cast<int64_t>(A2 * P.w1[f][1] + A3 * P.w2[f][1]) + A4 * static_cast<int64_t>(P.w3[f][1]);
	win[2] += static_cast<int64_t>(A3 * P.w2[f][2]) + A4 * static_cast<int64_t>(P.w3[f][2]);
	win[3] += static_cast<int64_t>(A3 * P.w2[f][3]) + A4 * static_cast<int64_t>(P.w3[f][3]);
	win[4] += A4 * static_cast<int64_t>(P.w3[f][4]);
}

// Adds the CRT value of one packed coefficient (residues x[4]) times f to the
// window at positions 0..4.
__device__ __forceinline__ void crt_window(const uint32_t x[4], int dup, const PackK &P, int64_t (&win)[7])
{
	uint32_t g[4] = { x[0], x[1], x[2], x[3] };
	crt_garner4(g);
	crt_window_g(g, dup, P, win);
}

// Completes the digit at window position 0 and shifts the window by one.
__device__ __forceinline__ int32_t window_digit(const CarryK &K, int64_t (&win)[7])
{
	int64_t q;
	const int32_t d = carry_wide(win[0], K, q);
#pragma unroll
	for (int j = 0; j < 6; ++j) win[j] = win[j + 1];
	win[6] = 0;
	win[0] += q;
	return d;
}

// Adds a packed segment carry (c[k] at digit k, k < 5) to D consecutive
// digits, reducing until the running carry is 0 or +-1, which stays in the
// next digit unreduced (|digit| <= b/2 + 1); false if the carry did not fit.
template <int D>
__device__ __forceinline__ bool absorb5(int32_t (&dg)[D], const int64_t (&c)[PK_CARRY], const CarryK &K)
{
	int64_t q = 0;
	bool done = false;
#pragma unroll
	for (int k = 0; k < D; ++k)
	{
		if (done) continue;
		const int64_t in = (k < PK_CARRY) ? c[k] : 0;
		if ((k >= PK_CARRY) && (q >= -1) && (q <= 1))
		{
			dg[k] += static_cast<int32_t>(q);
			q = 0;
			done = true;
			continue;
		}
		dg[k] = carry_wide(static_cast<int64_t>(dg[k]) + in + q, K, q);
	}
	return done || (q == 0);
}

}  // namespace gfc
