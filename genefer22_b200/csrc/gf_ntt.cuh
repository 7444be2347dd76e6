// gf_ntt.cuh -- negacyclic number-theoretic transform building blocks.
//
// The transform of length N = 2^n evaluates a digit polynomial at the N
// roots of X^N + 1 (the same quotient ring genefer squares in,
// src/transformCPUi32.h:691-715 and ocl/kernel.cl).  Forward: Cooley-Tukey
// butterflies (a, b) -> (a + w b, a - w b); inverse: Gentleman-Sande
// (a, b) -> (a + b, (a - b) / w).  At global stage s (0 <= s < n) element j
// pairs with j + N/2^(s+1) and uses the root table entry
//     idx = 2^s + (j >> (n - s)),   W[idx] = psi^bitrev_n(idx)
// where psi is a primitive 2N-th root of unity.  A sub-transform that covers
// the stages [s0, s0 + l) of one contiguous block of the global index space
// is described by its `base` (the block number at stage s0): a column pass of
// the four-step decomposition has base 1, row k of a row pass has base R + k.
//
// Inside a pass, r consecutive stages are done in registers on groups of 2^r
// elements (radix 2^r); groups are staged through shared memory between
// passes.
#pragma once

#include "gf_arith.cuh"

namespace gfc {

// f(integral_constant<B>), ..., f(integral_constant<E - 1>): a loop whose index
// is a compile-time constant in every iteration.
template <int B, int E, class F>
__device__ __forceinline__ void static_for(F &&f)
{
	if constexpr (B < E)
	{
		f(std::integral_constant<int, B>{});
		static_for<B + 1, E>(f);
	}
}

// Z: arithmetic of one prime (Zp with the prime as a constant, or ZpR with
// the prime in registers); R: its root type (Z::root_t).
template <class Z, class R>
__device__ __forceinline__ void bfly_ct(const Z &z, uint32_t &a, uint32_t &b, R w)
{
	const uint32_t t = z.mulr(b, w);
	b = z.sub(a, t);
	a = z.add(a, t);
}

template <class Z, class R>
__device__ __forceinline__ void bfly_gs(const Z &z, uint32_t &a, uint32_t &b, R wi)
{
	const uint32_t t = z.sub(a, b);
	a = z.add(a, b);
	b = z.mulr(t, wi);
}

// Root tables: entry idx of a table is one word (RootM: Montgomery form, the
// 32-bit primes) or two words at 2 idx, 2 idx + 1 (RootS: the root and its
// Shoup quotient, the 31-bit primes); entry 0 holds the normalisation
// constant (word 0, Montgomery form, for the Montgomery product).
//
// The twiddles of one radix-2^r group: w[2^t - 1 + sb] = entry (tbase << t) + sb
// for stage t < r of the group and sb < 2^t.  The 2^t entries of stage t are
// consecutive and start at a multiple of 2^t entries, so they load as 16-byte
// vectors (one 8-byte vector for the smallest stages; tables start on 32-byte
// boundaries).
template <int r>
__device__ __forceinline__ void load_twiddles(RootM (&w)[(1 << r) - 1], uint32_t tbase, const uint32_t *__restrict__ tw)
{
#pragma unroll
	for (int t = 0; t < r; ++t)
	{
		const uint32_t *p = tw + (static_cast<size_t>(tbase) << t);
		if (t >= 2)
		{
#pragma unroll
			for (int v = 0; v < (1 << t) / 4; ++v)
			{
				const uint4 u = __ldg(reinterpret_cast<const uint4 *>(p) + v);
				w[(1 << t) - 1 + 4 * v].w = u.x; w[(1 << t) + 4 * v].w = u.y;
				w[(1 << t) + 1 + 4 * v].w = u.z; w[(1 << t) + 2 + 4 * v].w = u.w;
			}
		}
		else if (t == 1)
		{
			const uint2 u = __ldg(reinterpret_cast<const uint2 *>(p));
			w[1].w = u.x; w[2].w = u.y;
		}
		else w[0].w = __ldg(p);
	}
}

template <int r>
__device__ __forceinline__ void load_twiddles(RootS (&w)[(1 << r) - 1], uint32_t tbase, const uint32_t *__restrict__ tw)
{
#pragma unroll
	for (int t = 0; t < r; ++t)
	{
		const uint32_t *p = tw + (static_cast<size_t>(tbase) << (t + 1));
		if (t >= 1)
		{
#pragma unroll
			for (int v = 0; v < (1 << t) / 2; ++v)
			{
				const uint4 u = __ldg(reinterpret_cast<const uint4 *>(p) + v);
				w[(1 << t) - 1 + 2 * v] = RootS{ u.x, u.y };
				w[(1 << t) + 2 * v] = RootS{ u.z, u.w };
			}
		}
		else
		{
			const uint2 u = __ldg(reinterpret_cast<const uint2 *>(p));
			w[0] = RootS{ u.x, u.y };
		}
	}
}

// r forward stages on 2^r registers.  Stage t of the group uses the table
// entries (tbase << t) + sb, sb < 2^t, with tbase = (base << sigma) + blk.
// All 2^r - 1 roots are loaded before the first butterfly.
template <class Z, int r>
__device__ __forceinline__ void fwd_reg(const Z &z, uint32_t (&x)[1 << r], uint32_t tbase, const uint32_t *__restrict__ tw)
{
	typename Z::root_t w[(1 << r) - 1];
	load_twiddles<r>(w, tbase, tw);
#pragma unroll
	for (int t = 0; t < r; ++t)
	{
		const int half = 1 << (r - 1 - t);
#pragma unroll
		for (int sb = 0; sb < (1 << t); ++sb)
#pragma unroll
			for (int m = 0; m < half; ++m)
				bfly_ct(z, x[sb * 2 * half + m], x[sb * 2 * half + m + half], w[(1 << t) - 1 + sb]);
	}
}

// r inverse stages (reverse order).  When `norm` is set the group contains
// global stage 0 (tbase == 1): its butterflies also multiply both outputs by
// the normalisation, a' = (a + b) c, b' = (a - b) K, with c = fw[0] and
// K = iv[0] prepared on the host.
template <class Z, int r>
__device__ __forceinline__ void inv_reg(const Z &z, uint32_t (&x)[1 << r], uint32_t tbase, const uint32_t *__restrict__ twi,
										bool norm, uint32_t c_norm, uint32_t k_norm)
{
	typename Z::root_t w[(1 << r) - 1];
	load_twiddles<r>(w, tbase, twi);
	static_for<0, r>([&](auto Q) {
		constexpr int t = r - 1 - decltype(Q)::value;
		constexpr int half = 1 << (r - 1 - t);
		if ((t == 0) && norm)
		{
#pragma unroll
			for (int m = 0; m < half; ++m)
			{
				uint32_t &a = x[m], &b = x[m + half];
				const uint32_t d = z.sub(a, b);
				a = z.mul(z.add(a, b), c_norm);
				b = z.mul(d, k_norm);
			}
		}
		else
		{
#pragma unroll
			for (int sb = 0; sb < (1 << t); ++sb)
#pragma unroll
				for (int m = 0; m < half; ++m)
					bfly_gs(z, x[sb * 2 * half + m], x[sb * 2 * half + m + half], w[(1 << t) - 1 + sb]);
		}
	});
}

// fwd_reg / inv_reg on two arrays that share their roots (the same row of two
// tests): the roots are loaded once, and each stage's butterflies alternate
// between the arrays, two independent chains.  No normalisation (rows never
// contain global stage 0).
template <class Z, int r>
__device__ __forceinline__ void fwd_reg2(const Z &z, uint32_t (&x)[1 << r], uint32_t (&y)[1 << r], uint32_t tbase,
										 const uint32_t *__restrict__ tw)
{
	typename Z::root_t w[(1 << r) - 1];
	load_twiddles<r>(w, tbase, tw);
#pragma unroll
	for (int t = 0; t < r; ++t)
	{
		const int half = 1 << (r - 1 - t);
#pragma unroll
		for (int sb = 0; sb < (1 << t); ++sb)
#pragma unroll
			for (int m = 0; m < half; ++m)
			{
				bfly_ct(z, x[sb * 2 * half + m], x[sb * 2 * half + m + half], w[(1 << t) - 1 + sb]);
				bfly_ct(z, y[sb * 2 * half + m], y[sb * 2 * half + m + half], w[(1 << t) - 1 + sb]);
			}
	}
}

template <class Z, int r>
__device__ __forceinline__ void inv_reg2(const Z &z, uint32_t (&x)[1 << r], uint32_t (&y)[1 << r], uint32_t tbase,
										 const uint32_t *__restrict__ twi)
{
	typename Z::root_t w[(1 << r) - 1];
	load_twiddles<r>(w, tbase, twi);
	static_for<0, r>([&](auto Q) {
		constexpr int t = r - 1 - decltype(Q)::value;
		constexpr int half = 1 << (r - 1 - t);
#pragma unroll
		for (int sb = 0; sb < (1 << t); ++sb)
#pragma unroll
			for (int m = 0; m < half; ++m)
			{
				bfly_gs(z, x[sb * 2 * half + m], x[sb * 2 * half + m + half], w[(1 << t) - 1 + sb]);
				bfly_gs(z, y[sb * 2 * half + m], y[sb * 2 * half + m + half], w[(1 << t) - 1 + sb]);
			}
	});
}

// Shared-memory address maps.  addr(i, lane) places element i of transform
// `lane`; off(m, step) is the address offset of element i0 + m step from
// element i0 for the groups the passes form (where it is independent of i0).
// Rows: transforms of length 2^L stored back to back, one padding word per 32.
// In a pass group either step >= 32, or i0 mod 32 + m step stays below 32,
// so the padding term is linear in m.
template <int L>
struct RowMap
{
	__device__ __forceinline__ static int addr(int i, int lane)
	{
		const int a = (lane << L) + i;
		return a + (a >> 5);
	}
	__host__ __device__ static constexpr int off(int m, int step) { return m * step + ((m * step) >> 5); }
};
// Columns: tile [2^l][RS] with the transform index i on the slow axis and
// one padding word after every 16 columns, so that both a warp reading 32
// consecutive columns and a warp reading one 16-digit segment per thread are
// free of bank conflicts.
template <int RS>
struct ColMap
{
	__device__ __forceinline__ static int addr(int i, int lane) { return i * RS + lane + (lane >> 4); }
	__host__ __device__ static constexpr int off(int m, int step) { return m * step * RS; }
};

// Group geometry of a radix-2^r pass at local stage sigma of a length-2^l
// transform: group g covers the elements
//   i_m = (blk << (l - sigma)) + o + (m << (l - sigma - r)),  m < 2^r,
// with blk = g >> (l - sigma - r), o = g mod 2^(l - sigma - r).
struct Group
{
	int i0, step, blk;
	__device__ __forceinline__ Group(int g, int l, int sigma, int r)
	{
		const int sh = l - sigma - r;
		blk = g >> sh;
		i0 = (blk << (l - sigma)) + (g & ((1 << sh) - 1));
		step = 1 << sh;
	}
};

}  // namespace gfc
