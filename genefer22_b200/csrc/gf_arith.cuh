// gf_arith.cuh -- exact modular and multi-word integer arithmetic for the
// B200 modular-squaring engine (integer pipe only; no floating point).
//
// Two RNS prime sets (one is chosen per test from b and n):
//   set 0: W = 2 primes just below 2^32  (widest exact range for two planes)
//   set 1: W = 3 primes just below 2^31  (every 12 <= n <= 23, b < 2^31;
//          31-bit primes let add/sub/Montgomery use min() corrections)
// The primes are the NTT-friendly primes genefer's transforms use
// (src/transformCPUi32.h:19-21 and src/transformGPU.h:37-105: 125*2^25+1,
// 243*2^24+1; 127*2^24+1, 63*2^25+1, 15*2^27+1).  Every product below is a
// Montgomery product with R = 2^32 (Montgomery 1985); residues are always
// fully reduced to [0, p).
#pragma once

#include <cstdint>

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
	static constexpr uint32_t p[3] = { 125u * (1u << 25) + 1u, 243u * (1u << 24) + 1u, 0u };
};

template <> struct PrimeSet<1>
{
	static constexpr int W = 3;
	static constexpr bool P31 = true;
	static constexpr uint32_t p[3] = { 127u * (1u << 24) + 1u, 63u * (1u << 25) + 1u, 15u * (1u << 27) + 1u };
};

// ---------------------------------------------------------------- Zp (one prime)

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

	// signed digit -> residue (|d| < p)
	__device__ __forceinline__ static uint32_t from_int(int32_t d)
	{
		return static_cast<uint32_t>(d) + ((d < 0) ? P : 0u);
	}
};

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
	static constexpr uint32_t p1 = PrimeSet<1>::p[0], p2 = PrimeSet<1>::p[1], p3 = PrimeSet<1>::p[2];
	static constexpr uint32_t c12 = to_mont_c(invmod_c(p1 % p2, p2), p2);                                   // p1^{-1} mod p2
	static constexpr uint32_t p1m3 = to_mont_c(p1 % p3, p3);                                                 // p1 mod p3
	static constexpr uint32_t c123 = to_mont_c(invmod_c(static_cast<uint32_t>((static_cast<uint64_t>(p1) * p2) % p3), p3), p3);   // (p1 p2)^{-1} mod p3
};

// The centred integer v with |v| < M/2 from its residues (normal form).
template <int SET>
__device__ __forceinline__ i128 crt(const uint32_t x[3]);

template <>
__device__ __forceinline__ i128 crt<0>(const uint32_t x[3])
{
	using C = Crt<0>;
	using Z2 = Zp<C::p2, false>;
	const uint32_t x1m2 = (x[0] >= C::p2) ? x[0] - C::p2 : x[0];
	const uint32_t a2 = Z2::mul(Z2::sub(x[1], x1m2), C::c12);
	const uint64_t v = static_cast<uint64_t>(a2) * C::p1 + x[0];
	constexpr uint64_t M = static_cast<uint64_t>(C::p1) * C::p2;
	return (v > M / 2) ? static_cast<i128>(v) - static_cast<i128>(M) : static_cast<i128>(v);
}

template <>
__device__ __forceinline__ i128 crt<1>(const uint32_t x[3])
{
	using C = Crt<1>;
	using Z2 = Zp<C::p2, true>;
	using Z3 = Zp<C::p3, true>;
	const uint32_t x1m2 = (x[0] >= C::p2) ? x[0] - C::p2 : x[0];
	const uint32_t a2 = Z2::mul(Z2::sub(x[1], x1m2), C::c12);
	// a3 = (x3 - x1 - a2 p1) / (p1 p2) mod p3
	const uint32_t x1m3 = (x[0] >= C::p3) ? x[0] - C::p3 : x[0];
	const uint32_t t = Z3::add(x1m3, Z3::mul(a2, C::p1m3));
	const uint32_t a3 = Z3::mul(Z3::sub(x[2], t), C::c123);
	// v = x1 + p1 (a2 + p2 a3)
	const uint64_t h = static_cast<uint64_t>(a3) * C::p2 + a2;
	const u128 v = static_cast<u128>(h) * C::p1 + x[0];
	constexpr u128 M = static_cast<u128>(static_cast<uint64_t>(C::p1) * C::p2) * C::p3;
	return (v > M / 2) ? static_cast<i128>(v) - static_cast<i128>(M) : static_cast<i128>(v);
}

// ---------------------------------------------------------------- base-b digit extraction

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

// Balanced digit of s in [-b/2, b/2) and carry floor((s + b/2) / b),
// for |s| < 2^95 (b even; for odd b the digit lies in [-(b-1)/2, (b+1)/2)).
__device__ __forceinline__ int32_t digit_carry(i128 s, uint32_t b, uint64_t binv, int64_t &carry)
{
	const uint32_t h = b / 2;
	const i128 t = s + h;
	const bool neg = (t < 0);
	const u128 a = static_cast<u128>(neg ? ~t : t);   // -t-1 when negative
	const uint64_t lo = static_cast<uint64_t>(a), hi = static_cast<uint64_t>(a >> 64);
	uint64_t r1, r0;
	const uint64_t q1 = divb64((hi << 32) | (lo >> 32), b, binv, r1);
	const uint64_t q0 = divb64((r1 << 32) | (lo & 0xffffffffu), b, binv, r0);
	uint64_t q = (q1 << 32) + q0;
	uint32_t r = static_cast<uint32_t>(r0);
	if (neg) { q = ~q; r = b - 1 - r; }
	carry = static_cast<int64_t>(q);
	return static_cast<int32_t>(r) - static_cast<int32_t>(h);
}

// Same for a 64-bit signed value (used when absorbing a carry into a digit).
__device__ __forceinline__ int32_t digit_carry64(int64_t s, uint32_t b, uint64_t binv, int64_t &carry)
{
	return digit_carry(static_cast<i128>(s), b, binv, carry);
}

}  // namespace gfc
