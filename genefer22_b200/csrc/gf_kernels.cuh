// gf_kernels.cuh -- sm_100a kernels of the modular-squaring engine.
//
// One squaring r <- r^2 (or 2 r^2) mod (b^N + 1), N = 2^n, is: digits ->
// residues in W prime planes -> forward negacyclic NTT -> pointwise square
// -> inverse NTT (normalisation folded into the last stage) -> CRT ->
// base-b carry.  This is the work of genefer's transform::squareDup
// (src/transform.h:59; CPU reference src/transformCPUi32.h:857-868).
//
// Resting state of a register: N signed int32 digits in natural order with
// |d| <= b/2 + 1 (balanced).  Kernel shapes:
//   * k_small (n <= 14): one CTA owns one test; the W planes live in shared
//     memory and the CTA can run many squarings without touching HBM.
//   * k_cluster: one test in the shared memory of a thread-block cluster.
//   * four-step: N = R x C.  The column-forward kernel (k_colr_fwd, k_col_fwd)
//     does the first log2 R stages, k_row the remaining stages + pointwise +
//     inverse on rows, the column-inverse kernel the last inverse stages, CRT
//     and the carry inside 16-digit segments (each segment's carry is added
//     to the next by the next column-forward pass, or by k_fixup).
//   * six-step: the column transform is split into a 16-point register pass
//     and a middle pass (k_midr, k_mid).
//   * packed digits (prime set 2): two digits per coefficient of a transform
//     of N/2 points over four primes (k_pcol_fwd, k_row, k_pcol_inv).
// Column kernels come in a one-thread-per-column form and a plane-split form
// (_s: a thread per plane and column) for launches that would leave SMs idle.
// Every kernel serves all tests of a batch in one launch; each CTA picks the
// code path of its test's prime set (W = 2, 3 or 4).
#pragma once

#include <type_traits>
#include <cooperative_groups.h>
#include "gf_ntt.cuh"

namespace gfc {

enum : int { OP_SQUARE = 0, OP_MUL = 1, OP_FWD = 2 };
enum : int { DUP_NONE = 0, DUP_ALL = 1, DUP_BITS = 2 };
enum : int { PM_FWD = 0, PM_INV = 1, PM_MID_SQ = 2, PM_MID_MUL = 3 };

constexpr int SEG = 16;          // digits per carry segment
constexpr int SMALL_MAX_LOGN = 14;
constexpr int WMAX = 3;

struct TestDesc
{
	int32_t *regs;          // num_regs x N digits
	uint32_t *planes;       // 3 x N transform scratch
	uint32_t *zp;           // 3 x N multiplicand (transform domain, normal form)
	int64_t *carry;         // N / SEG segment carries
	const uint32_t *ebits;  // exponent bits, bit i in word i/32 (may be null)
	uint64_t ewords;        // words ebits holds (0 with ebits null)
	CarryK ck;              // constants of the fused CRT + carry for this b
	PackK pk;               // packed-digit constants (set 2)
	uint32_t b;
	int32_t set;            // prime set: 0 (W = 2), 1 (W = 3), 2 (W = 4, packed digits)
};

// Root tables per prime (entries as load_twiddles reads them: one word in
// Montgomery form for 32-bit primes, root and Shoup quotient for 31-bit
// primes); word 0 of fw is the normalisation c, word 0 of iv the constant K
// of the last inverse stage, both in Montgomery form.
struct Tables
{
	const uint32_t *fw[4];  // forward roots
	const uint32_t *iv[4];  // inverse roots
	const uint32_t *tf[4];  // six-step twist factors, forward (twist_regs), of the batch's split
	const uint32_t *ti[4];  // and inverse
};

struct Args
{
	const TestDesc *desc;   // all tests of the batch
	const int32_t *tests;   // indices of the tests this launch serves
	int64_t *pos;           // per-test current exponent bit index
	uint32_t *err;          // error flags (bit 0: carry not absorbed)
	Tables tab[3];          // root tables of prime sets 0, 1 (length N) and 2 (length N/2)
	int n, lr;              // log2 N, log2 R (four-step)
	int num_regs, src, dst; // registers
	int op, dup_mode, count, j;  // operation, dup source, squarings (k_small), squaring index in block
	int fix;                // four-step column-forward: register src has pending segment carries
	int pdl_graph;          // host only: graph-captured launches keep programmatic edges
	int twist;              // six-step: the middle pass twists, every row transform has base 1
	uint32_t ntests;        // tests of the batch (0: unchecked); the guard of test_ok
};

template <int SET, int PL>
using ZS = Zp<PrimeSet<SET>::p[PL], PrimeSet<SET>::P31>;

template <int SET, class F>
__device__ __forceinline__ void for_planes(F &&f)
{
	f(std::integral_constant<int, 0>{});
	f(std::integral_constant<int, 1>{});
	if constexpr (PrimeSet<SET>::W >= 3) f(std::integral_constant<int, 2>{});
	if constexpr (PrimeSet<SET>::W >= 4) f(std::integral_constant<int, 3>{});
}



__device__ __forceinline__ bool exp_bit(const uint32_t *ebits, int64_t i)
{
	return ((__ldg(&ebits[i >> 5]) >> (i & 31)) & 1u) != 0;
}

// Error word bits: 1 a segment carry not absorbed, 2 a guard (below) tripped.
constexpr uint32_t ERR_CARRY = 1u, ERR_GUARD = 2u;

// The guard of every kernel that takes a test from the launch's list: the
// test index lies in the batch (with dup_bit below, the exponent position in
// the test's exponent words).  A corrupted list would otherwise make the
// kernel touch memory it does not own; instead the guard records ERR_GUARD
// (reported by the next synchronising call) and the test is skipped.  Checked
// when the launch carries the batch's size (a.ntests != 0).  Measured on one
// B200: 0.4 % of a 64-test n = 16 squaring (89.8 -> 90.2 us); checking every
// descriptor pointer against the batch's allocation as well (four more loads
// per CTA) cost 2.9 %.
__device__ __forceinline__ bool test_ok(const Args &a, int t)
{
	const bool ok = (a.ntests == 0) || (static_cast<uint32_t>(t) < a.ntests);
	if (!ok) atomicOr(a.err, ERR_GUARD);
	return ok;
}

// Exponent bit i of test d, guarded: a position beyond the test's exponent
// words records ERR_GUARD and reads as 0.
__device__ __forceinline__ bool dup_bit(const Args &a, const TestDesc &d, int64_t i)
{
	if ((d.ebits == nullptr) || (static_cast<uint64_t>(i >> 5) >= d.ewords))
	{
		atomicOr(a.err, ERR_GUARD);
		return false;
	}
	return exp_bit(d.ebits, i);
}

// Programmatic dependent launch: a kernel launched with programmatic stream
// serialization may be scheduled while the previous kernel of its stream is
// still running; it waits here (griddepcontrol.wait returns once every
// prerequisite grid has completed and its memory is visible, at once without
// one) before it touches memory, then lets the next kernel of the stream be
// scheduled as its own CTAs retire.  Every kernel starts with this.
__device__ __forceinline__ void pdl_wait()
{
	asm volatile("griddepcontrol.wait;" ::: "memory");
	asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// dup flag of squaring j (DUP_BITS: bit pos - j of the exponent); false with
// `active` cleared when the test has no squaring left.
__device__ __forceinline__ bool get_dup(const Args &a, const TestDesc &d, int t, int j, bool &active)
{
	active = test_ok(a, t);
	if (!active) return false;
	if (a.dup_mode == DUP_BITS)
	{
		const int64_t i = a.pos[t] - j;
		if (i < 0) { active = false; return false; }
		return dup_bit(a, d, i);
	}
	return a.dup_mode == DUP_ALL;
}

// Adds carry `c` to the digits of one segment: reduces while |c| > 1, then
// leaves the last +-1 in the next digit unreduced (|digit| <= b/2 + 1).
// `touched` receives the number of leading digits that changed; returns
// false if the carry did not fit in the segment.
template <int D>
__device__ __forceinline__ bool absorb(int32_t (&dg)[D], int64_t c, const CarryK &K, int &touched)
{
	bool active = (c != 0);
	touched = 0;
#pragma unroll
	for (int k = 0; k < D; ++k)
	{
		if (active)
		{
			touched = k + 1;
			if ((c > 1) || (c < -1))
			{
				dg[k] = carry_small(static_cast<int64_t>(dg[k]) + c, K, c);
			}
			else
			{
				dg[k] += static_cast<int32_t>(c);
				active = false;
			}
		}
	}
	return !active;
}

template <int D>
__device__ __forceinline__ bool absorb(int32_t (&dg)[D], int64_t c, const CarryK &K)
{
	int touched;
	return absorb<D>(dg, c, K, touched);
}

// Carry into segment s (16 digits) of a register with N / SEG segments.
// Takes the pending carry into segment s (negated across the wrap).  With
// `clear` it is also cleared, so that a test which sits out later squarings of
// its batch (DUP_BITS, position below 0) never has it applied twice: needed
// where nothing overwrites the carries after the absorption (the stand-alone
// fix-ups, a forward transform of a multiplicand, a cluster loading a test);
// a squaring or product rewrites every carry of every test it absorbs for.
__device__ __forceinline__ int64_t take_carry(const TestDesc &d, size_t s, size_t nseg, bool clear = true)
{
	int64_t *const p = (s == 0) ? &d.carry[nseg - 1] : &d.carry[s - 1];
	const int64_t c = *p;
	if (clear && (c != 0)) *p = 0;
	return (s == 0) ? -c : c;
}

__device__ __forceinline__ void fix_segment(const TestDesc &d, int32_t *seg, int istride, int32_t *g, int64_t cin,
											uint32_t *err)
{
	if (cin == 0) return;
	int32_t dg[SEG];
#pragma unroll
	for (int i = 0; i < SEG; ++i) dg[i] = seg[i * istride];
	int touched;
	if (!absorb<SEG>(dg, cin, d.ck, touched)) atomicOr(err, 1u);
#pragma unroll
	for (int i = 0; i < SEG; ++i)
		if (i < touched) { seg[i * istride] = dg[i]; g[i] = dg[i]; }
}

// Radix schedule of a length-2^L transform: passes of 4 stages starting at
// stage 4p; the last pass takes the remainder.
template <int L>
struct Sched
{
	static constexpr int NP = (L + 3) / 4;
	__host__ __device__ static constexpr int r(int p) { return (p < L / 4) ? 4 : (L % 4); }
	__host__ __device__ static constexpr int s(int p) { return 4 * p; }
};

// Balanced schedule: as few passes as Sched, their radices differing by one at
// most, the larger ones last (2^9: 3, 3, 3; 2^10: 3, 3, 4; 2^11: 3, 4, 4), so
// that the groups of every pass but the last are 8 points.
template <int L>
struct SchedB
{
	static constexpr int NP = (L + 3) / 4;
	static constexpr int LO = L / NP, HI = NP - L % NP;   // passes p >= HI take LO + 1 stages
	__host__ __device__ static constexpr int r(int p) { return LO + ((p >= HI) ? 1 : 0); }
	__host__ __device__ static constexpr int s(int p) { return LO * p + ((p > HI) ? p - HI : 0); }
};

// Every pass of a schedule starts where the one before it ends, and the
// passes cover the L stages.
template <class SC, int L>
constexpr bool sched_covers()
{
	int at = 0;
	for (int p = 0; p < SC::NP; ++p)
	{
		if ((SC::s(p) != at) || (SC::r(p) < 1) || (SC::r(p) > 4)) return false;
		at += SC::r(p);
	}
	return at == L;
}
static_assert(sched_covers<SchedB<8>, 8>() && sched_covers<SchedB<9>, 9>() && sched_covers<SchedB<10>, 10>() &&
				  sched_covers<SchedB<11>, 11>() && sched_covers<SchedB<13>, 13>(),
			  "balanced radix schedule");

// ------------------------------------------------------------------ passes

// One radix-2^r pass over the W planes (pstride words apart) of a shared-memory
// tile holding 2^lanes_log transforms of length 2^l.  Work item = one group of
// one lane, all planes.  PM_FWD / PM_INV: r forward / inverse stages;
// PM_MID_SQ / PM_MID_MUL: r forward stages, pointwise square (or product with
// the multiplicand at zrow[PL * zstride + (lane << l) + i]), r inverse stages.
//
// With PSPLIT a work item is one group of one lane of one plane (items of a
// plane consecutive, so a warp keeps one prime), W times as many items.
//
// IO selects where the group's elements come from and go to: IO_SMEM both in
// the tile; IO_GIN loads from global memory (gmem + pl gstride + (lane << L) + i,
// natural order) and stores to the tile; IO_GOUT loads from the tile and
// stores to global memory.  The first forward and the last inverse pass of a
// row read and write the planes in global memory directly (a warp takes 32
// consecutive groups, so each of its 2^r accesses is one coalesced line).
enum : int { IO_SMEM = 0, IO_GIN = 1, IO_GOUT = 2 };

template <int SET, int r, int MODE, int L, int SIGMA, class Map, int IO = IO_SMEM, bool PSPLIT = false, bool NORM = true>
__device__ __forceinline__ void pass_all(uint32_t *buf, int pstride, int lanes_log, bool lane_fast, uint32_t base0,
										 uint32_t base_step, const Tables &tab, const uint32_t *__restrict__ zrow,
										 size_t zstride, uint32_t *gmem = nullptr, size_t gstride = 0, int pl_lo = 0,
										 int pl_hi = PrimeSet<SET>::W)
{
	constexpr int E = 1 << r;
	constexpr int GL = L - r;                 // log2 groups per transform
	constexpr int STEP = 1 << (L - SIGMA - r);
	const int per_log = lanes_log + GL;
	const int items = PSPLIT ? ((pl_hi - pl_lo) << per_log) : (1 << per_log);
	for (int it0 = threadIdx.x; it0 < items; it0 += blockDim.x)
	{
		int it = it0, p_first = pl_lo, p_end = pl_hi;
		if constexpr (PSPLIT)
		{
			p_first = pl_lo + (it0 >> per_log);
			p_end = p_first + 1;
			it = it0 & ((1 << per_log) - 1);
		}
		int lane, g;
		if (lane_fast) { lane = it & ((1 << lanes_log) - 1); g = it >> lanes_log; }
		else { g = it & ((1 << GL) - 1); lane = it >> GL; }
		const Group G(g, L, SIGMA, r);
		const uint32_t tb = ((base0 + static_cast<uint32_t>(lane) * base_step) << SIGMA) + G.blk;
		const int base = Map::addr(G.i0, lane);
#pragma unroll 1
		for (int pl = p_first; pl < p_end; ++pl)
		{
			const auto z = prime_rt<SET>(pl);
			uint32_t *pb = buf + (pl - pl_lo) * pstride + base;
			uint32_t *gb = gmem;
			if constexpr (IO != IO_SMEM) gb = gmem + pl * gstride + (static_cast<size_t>(lane) << L) + G.i0;
			uint32_t x[E];
			if constexpr (IO == IO_GIN)
			{
#pragma unroll
				for (int m = 0; m < E; ++m) x[m] = gb[m * STEP];
			}
			else
			{
#pragma unroll
				for (int m = 0; m < E; ++m) x[m] = pb[Map::off(m, STEP)];
			}
			if constexpr (MODE != PM_INV) fwd_reg<decltype(z), r>(z, x, tb, tab.fw[pl]);
			if constexpr (MODE == PM_MID_SQ)
			{
#pragma unroll
				for (int m = 0; m < E; ++m) x[m] = z.mul(x[m], x[m]);
			}
			if constexpr (MODE == PM_MID_MUL)
			{
				const uint32_t *zz = zrow + pl * zstride + (static_cast<size_t>(lane) << L) + G.i0;
#pragma unroll
				for (int m = 0; m < E; ++m) x[m] = z.mul(x[m], __ldg(&zz[m * STEP]));
			}
			if constexpr (MODE != PM_FWD)
				inv_reg<decltype(z), r>(z, x, tb, tab.iv[pl], NORM && (tb == 1u), __ldg(&tab.fw[pl][0]),
										__ldg(&tab.iv[pl][0]));
			if constexpr (IO == IO_GOUT)
			{
#pragma unroll
				for (int m = 0; m < E; ++m) gb[m * STEP] = x[m];
			}
			else
			{
#pragma unroll
				for (int m = 0; m < E; ++m) pb[Map::off(m, STEP)] = x[m];
			}
		}
	}
}

// Forward passes 0 .. NP-1 (or NP-2 with SKIP_LAST) of schedule SC, a barrier
// after each.
template <int SET, int L, bool SKIP_LAST, class Map, bool PSPLIT = false, class SC = Sched<L>>
__device__ __forceinline__ void run_fwd(uint32_t *buf, int pstride, int lanes_log, bool lane_fast, uint32_t base0,
										uint32_t base_step, const Tables &tab, int pl_lo = 0, int pl_hi = PrimeSet<SET>::W)
{
	constexpr int NP = SC::NP - (SKIP_LAST ? 1 : 0);
	static_for<0, NP>([&](auto P) {
		constexpr int p = decltype(P)::value;
		pass_all<SET, SC::r(p), PM_FWD, L, SC::s(p), Map, IO_SMEM, PSPLIT>(buf, pstride, lanes_log, lane_fast, base0,
																			base_step, tab, nullptr, 0, nullptr, 0,
																			pl_lo, pl_hi);
		__syncthreads();
	});
}

// Inverse passes NP-1 (or NP-2 with SKIP_LAST) .. 0.
template <int SET, int L, bool SKIP_LAST, class Map, bool PSPLIT = false, class SC = Sched<L>>
__device__ __forceinline__ void run_inv(uint32_t *buf, int pstride, int lanes_log, bool lane_fast, uint32_t base0,
										uint32_t base_step, const Tables &tab, int pl_lo = 0, int pl_hi = PrimeSet<SET>::W)
{
	constexpr int NP = SC::NP - (SKIP_LAST ? 1 : 0);
	static_for<0, NP>([&](auto Q) {
		constexpr int p = NP - 1 - decltype(Q)::value;
		pass_all<SET, SC::r(p), PM_INV, L, SC::s(p), Map, IO_SMEM, PSPLIT>(buf, pstride, lanes_log, lane_fast, base0,
																			base_step, tab, nullptr, 0, nullptr, 0,
																			pl_lo, pl_hi);
		__syncthreads();
	});
}

// Row transform of one row whose planes stay in global memory at g (plane
// stride gstride): the first forward pass reads them, the last inverse pass
// writes them, the passes between go through the shared-memory tile.
// Squaring or product only (not OP_FWD).  A row never holds global stage 0
// (its base is R + k, or 1 after a six-step twist), so no inverse pass
// normalises.
template <int SET, int L, class Map>
__device__ __forceinline__ void row_core_global(uint32_t *buf, int pstride, uint32_t base0, const Tables &tab,
												const uint32_t *zrow, size_t zstride, int op, uint32_t *g, size_t gstride,
												int pl_lo, int pl_hi)
{
	constexpr int NP = Sched<L>::NP;
	static_assert(NP >= 2, "rows of at least two passes");
	static_for<0, NP - 1>([&](auto P) {
		constexpr int p = decltype(P)::value;
		if constexpr (p == 0)
			pass_all<SET, Sched<L>::r(p), PM_FWD, L, 4 * p, Map, IO_GIN>(buf, pstride, 0, false, base0, 1u, tab, nullptr, 0,
																		  g, gstride, pl_lo, pl_hi);
		else
			pass_all<SET, Sched<L>::r(p), PM_FWD, L, 4 * p, Map>(buf, pstride, 0, false, base0, 1u, tab, nullptr, 0,
																  nullptr, 0, pl_lo, pl_hi);
		__syncthreads();
	});
	constexpr int PL = NP - 1;
	if (op == OP_MUL)
		pass_all<SET, Sched<L>::r(PL), PM_MID_MUL, L, 4 * PL, Map, IO_SMEM, false, false>(
			buf, pstride, 0, false, base0, 1u, tab, zrow, zstride, nullptr, 0, pl_lo, pl_hi);
	else
		pass_all<SET, Sched<L>::r(PL), PM_MID_SQ, L, 4 * PL, Map, IO_SMEM, false, false>(
			buf, pstride, 0, false, base0, 1u, tab, zrow, zstride, nullptr, 0, pl_lo, pl_hi);
	__syncthreads();
	static_for<0, NP - 1>([&](auto Q) {
		constexpr int p = NP - 2 - decltype(Q)::value;
		if constexpr (p == 0)
			pass_all<SET, Sched<L>::r(p), PM_INV, L, 4 * p, Map, IO_GOUT, false, false>(
				buf, pstride, 0, false, base0, 1u, tab, nullptr, 0, g, gstride, pl_lo, pl_hi);
		else
		{
			pass_all<SET, Sched<L>::r(p), PM_INV, L, 4 * p, Map, IO_SMEM, false, false>(
				buf, pstride, 0, false, base0, 1u, tab, nullptr, 0, nullptr, 0, pl_lo, pl_hi);
			__syncthreads();
		}
	});
}

// One radix-2^r pass of a row of plane pl for two tests at once (k_row2):
// the tests' tiles buf0, buf1 (or their rows in global memory g0, g1 for the
// first forward and the last inverse pass), the same roots.  MODE as in
// pass_all; lanes and plane splitting are not used.  `store1` false: the
// second lane duplicates the first test and writes only its own tile.
template <int SET, int r, int MODE, int L, int SIGMA, class Map, int IO>
__device__ __forceinline__ void pass_pair(uint32_t *buf0, uint32_t *buf1, uint32_t base0, const Tables &tab,
										  const uint32_t *__restrict__ zrow0, const uint32_t *__restrict__ zrow1,
										  uint32_t *g0, uint32_t *g1, int pl, bool store1)
{
	constexpr int E = 1 << r;
	constexpr int GL = L - r;
	constexpr int STEP = 1 << (L - SIGMA - r);
	const auto z = prime_rt<SET>(pl);
	for (int g = threadIdx.x; g < (1 << GL); g += blockDim.x)
	{
		const Group G(g, L, SIGMA, r);
		const uint32_t tb = (base0 << SIGMA) + G.blk;
		const int base = Map::addr(G.i0, 0);
		uint32_t x[E], y[E];
		if constexpr (IO == IO_GIN)
		{
#pragma unroll
			for (int m = 0; m < E; ++m) { x[m] = g0[G.i0 + m * STEP]; y[m] = g1[G.i0 + m * STEP]; }
		}
		else
		{
#pragma unroll
			for (int m = 0; m < E; ++m) { x[m] = buf0[base + Map::off(m, STEP)]; y[m] = buf1[base + Map::off(m, STEP)]; }
		}
		if constexpr (MODE != PM_INV) fwd_reg2<decltype(z), r>(z, x, y, tb, tab.fw[pl]);
		if constexpr (MODE == PM_MID_SQ)
		{
#pragma unroll
			for (int m = 0; m < E; ++m) { x[m] = z.mul(x[m], x[m]); y[m] = z.mul(y[m], y[m]); }
		}
		if constexpr (MODE == PM_MID_MUL)
		{
#pragma unroll
			for (int m = 0; m < E; ++m)
			{
				x[m] = z.mul(x[m], __ldg(&zrow0[G.i0 + m * STEP]));
				y[m] = z.mul(y[m], __ldg(&zrow1[G.i0 + m * STEP]));
			}
		}
		if constexpr (MODE != PM_FWD) inv_reg2<decltype(z), r>(z, x, y, tb, tab.iv[pl]);
		if constexpr (IO == IO_GOUT)
		{
#pragma unroll
			for (int m = 0; m < E; ++m) g0[G.i0 + m * STEP] = x[m];
			if (store1)
			{
#pragma unroll
				for (int m = 0; m < E; ++m) g1[G.i0 + m * STEP] = y[m];
			}
		}
		else
		{
#pragma unroll
			for (int m = 0; m < E; ++m) { buf0[base + Map::off(m, STEP)] = x[m]; buf1[base + Map::off(m, STEP)] = y[m]; }
		}
	}
}

// row_core_global for two tests (k_row2): squaring or product of row `base0`
// of plane pl, the rows in global memory at g0, g1, tiles buf0, buf1.
template <int SET, int L, class Map>
__device__ __forceinline__ void row_core_pair(uint32_t *buf0, uint32_t *buf1, uint32_t base0, const Tables &tab,
											  const uint32_t *zrow0, const uint32_t *zrow1, int op, uint32_t *g0,
											  uint32_t *g1, int pl, bool store1)
{
	constexpr int NP = Sched<L>::NP;
	static_assert(NP >= 2, "rows of at least two passes");
	static_for<0, NP - 1>([&](auto P) {
		constexpr int p = decltype(P)::value;
		if constexpr (p == 0)
			pass_pair<SET, Sched<L>::r(p), PM_FWD, L, 4 * p, Map, IO_GIN>(buf0, buf1, base0, tab, nullptr, nullptr, g0, g1,
																		   pl, store1);
		else
			pass_pair<SET, Sched<L>::r(p), PM_FWD, L, 4 * p, Map, IO_SMEM>(buf0, buf1, base0, tab, nullptr, nullptr,
																			nullptr, nullptr, pl, store1);
		__syncthreads();
	});
	constexpr int PL = NP - 1;
	if (op == OP_MUL)
		pass_pair<SET, Sched<L>::r(PL), PM_MID_MUL, L, 4 * PL, Map, IO_SMEM>(buf0, buf1, base0, tab, zrow0, zrow1, nullptr,
																			  nullptr, pl, store1);
	else
		pass_pair<SET, Sched<L>::r(PL), PM_MID_SQ, L, 4 * PL, Map, IO_SMEM>(buf0, buf1, base0, tab, nullptr, nullptr,
																			 nullptr, nullptr, pl, store1);
	__syncthreads();
	static_for<0, NP - 1>([&](auto Q) {
		constexpr int p = NP - 2 - decltype(Q)::value;
		if constexpr (p == 0)
			pass_pair<SET, Sched<L>::r(p), PM_INV, L, 4 * p, Map, IO_GOUT>(buf0, buf1, base0, tab, nullptr, nullptr, g0, g1,
																			pl, store1);
		else
		{
			pass_pair<SET, Sched<L>::r(p), PM_INV, L, 4 * p, Map, IO_SMEM>(buf0, buf1, base0, tab, nullptr, nullptr,
																			nullptr, nullptr, pl, store1);
			__syncthreads();
		}
	});
}

// Row transforms in shared memory: forward (OP_FWD), or forward + pointwise
// square / product + inverse.
template <int SET, int L, class Map, bool PSPLIT = false, class SC = Sched<L>>
__device__ __forceinline__ void row_core(uint32_t *buf, int pstride, int lanes_log, uint32_t base0, const Tables &tab,
										 const uint32_t *zrow, size_t zstride, int op)
{
	constexpr int PL = SC::NP - 1;
	if (op == OP_FWD) { run_fwd<SET, L, false, Map, PSPLIT, SC>(buf, pstride, lanes_log, false, base0, 1u, tab); return; }
	run_fwd<SET, L, true, Map, PSPLIT, SC>(buf, pstride, lanes_log, false, base0, 1u, tab);
	if (op == OP_MUL)
		pass_all<SET, SC::r(PL), PM_MID_MUL, L, SC::s(PL), Map, IO_SMEM, PSPLIT>(buf, pstride, lanes_log, false, base0,
																				  1u, tab, zrow, zstride);
	else
		pass_all<SET, SC::r(PL), PM_MID_SQ, L, SC::s(PL), Map, IO_SMEM, PSPLIT>(buf, pstride, lanes_log, false, base0,
																				 1u, tab, zrow, zstride);
	__syncthreads();
	run_inv<SET, L, true, Map, PSPLIT, SC>(buf, pstride, lanes_log, false, base0, 1u, tab);
}

// ------------------------------------------------------------------ k_small

// Single-CTA shape for one prime set: T0 threads own D = N / T0 digits each
// (CRT and carry).  With SPLIT (up to n = 12, for launches of fewer tests
// than SMs) the transform passes run plane-split, a thread per (plane,
// group), on T = W T0 threads: a lone test is one CTA on one SM, and W times
// the warps hide W times more latency.  MINB CTAs per SM bound the register
// budget.
template <int SET, int LOGN, bool SPLIT = false>
struct SmallShape
{
	static constexpr int W = PrimeSet<SET>::W;
	static constexpr int N = 1 << LOGN;
	static constexpr int PN = N + N / 32;                 // padded plane
	static constexpr int T0 = (LOGN <= 12) ? (N / 16) : 512;
	static constexpr bool PSPLIT = SPLIT && (LOGN <= 12);
	static constexpr int T = PSPLIT ? W * T0 : T0;
	static constexpr int MINB = (T <= 128) ? 4 : ((T <= 256) ? 2 : 1);
	static constexpr size_t SMEM = size_t(W) * PN * 4 + size_t(T) * 8;
};

template <int SET, int LOGN, bool SPLIT>
__device__ __forceinline__ void small_body(const Args &a, int t, const TestDesc &d, uint32_t *sm)
{
	using S = SmallShape<SET, LOGN, SPLIT>;
	constexpr int N = S::N, PN = S::PN, T = S::T, T0 = S::T0;
	constexpr int D = N / T0;          // digits per owner thread (multiple of SEG)
	static_assert(D % SEG == 0, "digits per thread");
	int64_t *const sc = reinterpret_cast<int64_t *>(sm + S::W * PN);
	const Tables &tab = a.tab[SET];
	const int tid = threadIdx.x;
	const bool owner = (tid < T0);     // threads T0 .. T-1 join the transform passes only
	using MP = RowMap<LOGN>;

	int32_t dg[D];
	if (owner)
	{
		const int4 *src = reinterpret_cast<const int4 *>(d.regs + static_cast<size_t>(a.src) * N + tid * D);
#pragma unroll
		for (int i = 0; i < D / 4; ++i)
		{
			const int4 v = src[i];
			dg[4 * i] = v.x; dg[4 * i + 1] = v.y; dg[4 * i + 2] = v.z; dg[4 * i + 3] = v.w;
		}
	}

	const int iters = (a.op == OP_SQUARE) ? a.count : 1;
	int done = 0;
	for (int it = 0; it < iters; ++it)
	{
		bool active = true;
		const bool dup = (a.op == OP_SQUARE) ? get_dup(a, d, t, it, active) : false;
		if (!active) break;

		if (owner)
		{
			for_planes<SET>([&](auto PLc) {
				constexpr int PL = decltype(PLc)::value;
				using Z = ZS<SET, PL>;
#pragma unroll
				for (int i = 0; i < D; ++i) sm[PL * PN + MP::addr(tid * D + i, 0)] = Z::from_int(dg[i]);
			});
		}
		__syncthreads();

		row_core<SET, LOGN, MP, S::PSPLIT>(sm, PN, 0, 1u, tab, d.zp, N, a.op);

		if (a.op == OP_FWD)
		{
#pragma unroll
			for (int pl = 0; pl < PrimeSet<SET>::W; ++pl)
				for (int i = tid; i < N; i += T) d.zp[pl * N + i] = sm[pl * PN + MP::addr(i, 0)];
			return;
		}

		// CRT + carry over each owner's D consecutive digits.
		if (owner)
		{
			int64_t c = 0;
#pragma unroll
			for (int i = 0; i < D; ++i)
			{
				uint32_t x[3];
#pragma unroll
				for (int pl = 0; pl < PrimeSet<SET>::W; ++pl) x[pl] = sm[pl * PN + MP::addr(tid * D + i, 0)];
				dg[i] = crt_carry<SET>(x, dup ? 1 : 0, d.ck, c);
			}
			sc[tid] = c;
		}
		__syncthreads();
		if (owner)
		{
			const int64_t cin = (tid == 0) ? -sc[T0 - 1] : sc[tid - 1];
			if (!absorb<D>(dg, cin, d.ck)) atomicOr(a.err, 1u);
		}
		__syncthreads();
		++done;
	}

	if (owner)
	{
		int4 *dst = reinterpret_cast<int4 *>(d.regs + static_cast<size_t>(a.dst) * N + tid * D);
#pragma unroll
		for (int i = 0; i < D / 4; ++i) dst[i] = make_int4(dg[4 * i], dg[4 * i + 1], dg[4 * i + 2], dg[4 * i + 3]);
	}
	if ((tid == 0) && (a.op == OP_SQUARE) && (a.dup_mode == DUP_BITS)) a.pos[t] -= done;
}

// One CTA per test of prime set SET; shared memory SmallShape<SET, LOGN, SPLIT>::SMEM.
template <int SET, int LOGN, bool SPLIT>
__global__ void __launch_bounds__(SmallShape<SET, LOGN, SPLIT>::T, SmallShape<SET, LOGN, SPLIT>::MINB)
	k_small(const Args a)
{
	pdl_wait();
	extern __shared__ __align__(16) uint32_t sm[];
	const int t = a.tests[blockIdx.x];
	if (!test_ok(a, t)) return;
	small_body<SET, LOGN, SPLIT>(a, t, a.desc[t], sm);
}

// ------------------------------------------------------------------ k_cluster

// One test per thread-block cluster of Q = 2^LQ CTAs, resident in shared
// memory for many squarings.  The test is the four-step matrix of Q rows of
// C = 2^LC digits; CTA q holds row q (digits q C .. q C + C - 1).  Per
// squaring: the Q-point column transforms (stages 0 .. LQ-1, base 1) read and
// write the Q rows through distributed shared memory, each CTA transforms its
// row (stages LQ .. n-1 with base 2^LQ + q, pointwise square, inverse), the
// inverse column transforms fold in the normalisation, and every owner thread
// turns 16 consecutive digits of its row into balanced base-b digits (CRT +
// carry); the carry out of each 16-digit segment enters the next one (across
// CTAs, and negated from the last segment to the first: b^N = -1) before the
// next squaring.  Digits stay in registers between squarings; global memory
// is read when a test starts and written when it ends.  A persistent grid of
// clusters takes tests t = cluster, cluster + clusters, ...
//
// Rows of 2^13 (n = 15..17, LQ = 2..4) have one owner thread per segment and
// no more threads.  Shorter rows (n = 12..14, LC = 9..11) add plane-split
// threads: the transform passes (balanced schedule, 8-point groups) and column
// transforms run a thread per (plane, group), W C / 8 threads, so that a lone
// small test spread over 8 or 16 SMs keeps several warps on each and a thread
// takes one group per pass.
template <int LQ, int LC = 13>
struct ClusterShape
{
	static constexpr int Q = 1 << LQ;
	static constexpr int C = 1 << LC;
	static constexpr int PC = C + C / 32;                 // padded plane (RowMap)
	static constexpr bool PS = (LC <= 11);                // plane-split passes
	// digits per owner thread: 16 (one carry segment of the engine), or 8 for
	// the short rows, whose owners then run half as long a carry chain (the
	// carries inside the kernel are its own; every carry fits 8 digits for
	// b >= 1024, absorb() checks it)
	static constexpr int D = PS ? SEG / 2 : SEG;
	static constexpr int T0 = C / D;                      // owner threads
	static constexpr int T = PS ? WMAX * C / 8 : T0;
	static constexpr int MINB = PS ? 1 : 2;
	// planes, the owners' carries, and (PS) a fourth word per digit for the
	// two-stage CRT
	static constexpr size_t SMEM = size_t(WMAX) * PC * 4 + size_t(T0) * 8 + (PS ? size_t(PC) * 4 : 0);
	using SC = std::conditional_t<PS, SchedB<LC>, Sched<LC>>;
	static_assert(T <= 1024, "threads per CTA");
};

// Distributed shared memory by 32-bit shared::cluster addresses: the word at
// shared-memory address `a` of this CTA, in the CTA of cluster rank `rank`.
__device__ __forceinline__ uint32_t dsm_addr(uint32_t a, uint32_t rank)
{
	uint32_t r;
	asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
	return r;
}
__device__ __forceinline__ uint32_t dsm_ld(uint32_t a)
{
	uint32_t v;
	asm volatile("ld.shared::cluster.u32 %0, [%1];" : "=r"(v) : "r"(a) : "memory");
	return v;
}
__device__ __forceinline__ void dsm_st(uint32_t a, uint32_t v)
{
	asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(a), "r"(v) : "memory");
}

// Q-point column transform of column j of plane PL (prime arithmetic z).
template <int LQ, bool INV, class Z>
__device__ __forceinline__ void cluster_col(const Z &z, uint32_t a, const uint32_t *fw, const uint32_t *iv)
{
	constexpr int Q = 1 << LQ;
	uint32_t x[Q];
#pragma unroll
	for (int k = 0; k < Q; ++k) x[k] = dsm_ld(dsm_addr(a, k));
	if constexpr (!INV) fwd_reg<Z, LQ>(z, x, 1u, fw);
	else inv_reg<Z, LQ>(z, x, 1u, iv, true, __ldg(&fw[0]), __ldg(&iv[0]));
#pragma unroll
	for (int k = 0; k < Q; ++k) dsm_st(dsm_addr(a, k), x[k]);
}

// Q-point column transforms of the columns q C/Q .. (q+1) C/Q - 1, all planes
// (plane-split shapes: a work item per (plane, column)).
template <int SET, int LQ, int LC, bool INV>
__device__ __forceinline__ void cluster_cols(uint32_t *sm, int q, const Tables &tab)
{
	using S = ClusterShape<LQ, LC>;
	constexpr int Q = S::Q, CQ = S::C / Q;
	using MP = RowMap<LC>;
	const uint32_t base = static_cast<uint32_t>(__cvta_generic_to_shared(sm));
	if constexpr (S::PS)
	{
		constexpr int W = PrimeSet<SET>::W;
#pragma unroll 1
		for (int it = threadIdx.x; it < W * CQ; it += blockDim.x)
		{
			const int pl = it / CQ, j = it % CQ;
			const auto z = prime_rt<SET>(pl);
			const uint32_t a = base + 4u * static_cast<uint32_t>(pl * S::PC + MP::addr(q * CQ + j, 0));
			cluster_col<LQ, INV>(z, a, tab.fw[pl], tab.iv[pl]);
		}
	}
	else
	{
#pragma unroll 1
		for (int j = threadIdx.x; j < CQ; j += S::T)
		{
			const uint32_t off = base + 4u * static_cast<uint32_t>(MP::addr(q * CQ + j, 0));
			for_planes<SET>([&](auto PLc) {
				constexpr int PL = decltype(PLc)::value;
				using Z = ZS<SET, PL>;
				cluster_col<LQ, INV>(Z{}, off + 4u * PL * S::PC, tab.fw[PL], tab.iv[PL]);
			});
		}
	}
}

// One test of prime set SET on this cluster: `count` squarings (fewer when
// the exponent runs out), from register src to register dst.
template <int SET, int LQ, int LC>
__device__ __forceinline__ void cluster_test(const Args &a, int t, const TestDesc &d, uint32_t *sm, int q)
{
	namespace cg = cooperative_groups;
	using S = ClusterShape<LQ, LC>;
	constexpr int Q = S::Q, C = S::C, PC = S::PC, T0 = S::T0, D = S::D, W = PrimeSet<SET>::W;
	using MP = RowMap<LC>;
	int64_t *const sc = reinterpret_cast<int64_t *>(sm + WMAX * PC);
	cg::cluster_group cl = cg::this_cluster();
	const int tid = threadIdx.x;
	const bool owner = (tid < T0);
	const Tables &tab = a.tab[SET];
	const size_t N = size_t(C) * Q;
	const size_t nseg = N / SEG;

	// Every CTA of the cluster reads the position once, before the first
	// cluster barrier, so that all take the same number of squarings.
	const int64_t pos0 = (a.dup_mode == DUP_BITS) ? a.pos[t] : 0;
	int iters = a.count;
	if (a.dup_mode == DUP_BITS) iters = (pos0 + 1 < iters) ? static_cast<int>((pos0 < 0) ? 0 : pos0 + 1) : iters;

	int32_t dg[D];
	if (owner)
	{
		const size_t j0 = static_cast<size_t>(q) * C + static_cast<size_t>(tid) * D;
		const int4 *src = reinterpret_cast<const int4 *>(d.regs + static_cast<size_t>(a.src) * N + j0);
#pragma unroll
		for (int i = 0; i < D / 4; ++i)
		{
			const int4 v = src[i];
			dg[4 * i] = v.x; dg[4 * i + 1] = v.y; dg[4 * i + 2] = v.z; dg[4 * i + 3] = v.w;
		}
		if (a.fix && (j0 % SEG == 0))
		{
			const int64_t cin = take_carry(d, j0 / SEG, nseg);
			if (!absorb<D>(dg, cin, d.ck)) atomicOr(a.err, 1u);
		}
	}

	for (int it = 0; it < iters; ++it)
	{
		const bool dup = (a.dup_mode == DUP_BITS) ? dup_bit(a, d, pos0 - it) : (a.dup_mode == DUP_ALL);
		if (owner)
		{
			for_planes<SET>([&](auto PLc) {
				constexpr int PL = decltype(PLc)::value;
				using Z = ZS<SET, PL>;
#pragma unroll
				for (int i = 0; i < D; ++i) sm[PL * PC + MP::addr(tid * D + i, 0)] = Z::from_int(dg[i]);
			});
		}
		cl.sync();
		cluster_cols<SET, LQ, LC, false>(sm, q, tab);
		cl.sync();
		row_core<SET, LC, MP, S::PS, typename S::SC>(sm, PC, 0, (1u << LQ) + static_cast<uint32_t>(q), tab, nullptr, 0,
													  OP_SQUARE);
		cl.sync();
		cluster_cols<SET, LQ, LC, true>(sm, q, tab);
		cl.sync();
		if constexpr (S::PS)
		{
			// every thread takes digits j = tid, tid + T, ... through the part of
			// the CRT that needs no carry and leaves (u, t) in the digit's plane
			// words and ex; the owners then run their carry chains alone
			uint32_t *const ex = reinterpret_cast<uint32_t *>(sc + T0);
#pragma unroll 1
			for (int j = tid; j < C; j += S::T)
			{
				const int aj = MP::addr(j, 0);
				uint32_t x[3];
#pragma unroll
				for (int pl = 0; pl < W; ++pl) x[pl] = sm[pl * PC + aj];
				uint64_t u, tt;
				crt_split<SET>(x, dup ? 1 : 0, d.ck, u, tt);
				sm[aj] = static_cast<uint32_t>(u);
				sm[PC + aj] = static_cast<uint32_t>(u >> 32);
				sm[2 * PC + aj] = static_cast<uint32_t>(tt);
				ex[aj] = static_cast<uint32_t>(tt >> 32);
			}
			__syncthreads();
			if (owner)
			{
				int64_t c = 0;
#pragma unroll
				for (int i = 0; i < D; ++i)
				{
					const int aj = MP::addr(tid * D + i, 0);
					const uint64_t u = sm[aj] | (static_cast<uint64_t>(sm[PC + aj]) << 32);
					const uint64_t tt = sm[2 * PC + aj] | (static_cast<uint64_t>(ex[aj]) << 32);
					dg[i] = crt_chain(u, tt, d.ck, c);
				}
				sc[tid] = c;
			}
		}
		else if (owner)
		{
			int64_t c = 0;
#pragma unroll
			for (int i = 0; i < D; ++i)
			{
				uint32_t x[3];
#pragma unroll
				for (int pl = 0; pl < W; ++pl) x[pl] = sm[pl * PC + MP::addr(tid * D + i, 0)];
				dg[i] = crt_carry<SET>(x, dup ? 1 : 0, d.ck, c);
			}
			sc[tid] = c;
		}
		cl.sync();
		if (owner)
		{
			int64_t cin;
			if (tid > 0) cin = sc[tid - 1];
			else
			{
				const uint32_t qp = (q == 0) ? Q - 1 : q - 1;
				const uint32_t ra = dsm_addr(static_cast<uint32_t>(__cvta_generic_to_shared(sc + T0 - 1)), qp);
				const uint64_t lo = dsm_ld(ra), hi = dsm_ld(ra + 4);
				cin = static_cast<int64_t>(lo | (hi << 32));
				if (q == 0) cin = -cin;
			}
			if (!absorb<D>(dg, cin, d.ck)) atomicOr(a.err, 1u);
		}
	}

	if (owner)
	{
		const size_t j0 = static_cast<size_t>(q) * C + static_cast<size_t>(tid) * D;
		int4 *dst = reinterpret_cast<int4 *>(d.regs + static_cast<size_t>(a.dst) * N + j0);
#pragma unroll
		for (int i = 0; i < D / 4; ++i) dst[i] = make_int4(dg[4 * i], dg[4 * i + 1], dg[4 * i + 2], dg[4 * i + 3]);
	}
	if ((tid == 0) && (q == 0) && (a.dup_mode == DUP_BITS)) a.pos[t] = (pos0 - iters < -1) ? -1 : pos0 - iters;
}

// Persistent grid of clusters over the tests a.tests[0 .. ntests-1], of
// either prime set.
template <int LQ, int LC>
__global__ void __launch_bounds__(ClusterShape<LQ, LC>::T, ClusterShape<LQ, LC>::MINB) k_cluster(const Args a, int ntests)
{
	pdl_wait();
	namespace cg = cooperative_groups;
	using S = ClusterShape<LQ, LC>;
	extern __shared__ __align__(16) uint32_t sm[];
	cg::cluster_group cl = cg::this_cluster();
	const int q = static_cast<int>(cl.block_rank());
	const int ncl = gridDim.x / S::Q, cid = blockIdx.x / S::Q;
	for (int ti = cid; ti < ntests; ti += ncl)
	{
		const int t = a.tests[ti];
		if (test_ok(a, t))
		{
			const TestDesc &d = a.desc[t];
			if (d.set == 0) cluster_test<0, LQ, LC>(a, t, d, sm, q); else cluster_test<1, LQ, LC>(a, t, d, sm, q);
		}
		// the next test's first shared-memory writes follow this barrier, after
		// every CTA has read this test's last carries
		cl.sync();
	}
}

// ------------------------------------------------------------------ four-step

__host__ __device__ constexpr int ilog2c(int x) { return (x <= 1) ? 0 : 1 + ilog2c(x / 2); }
__host__ __device__ constexpr int col_width(int lr) { return (lr >= 10) ? 16 : ((4096 >> lr) > 32 ? (4096 >> lr) : 32); }

// Column tile: CW columns x R rows per plane, row stride RS (ColMap padding).
template <int LR>
struct ColShape
{
	static constexpr int R = 1 << LR;
	static constexpr int CW = col_width(LR);
	static constexpr int CWL = ilog2c(CW);
	static constexpr int RS = CW + ((CW / 16 > 1) ? CW / 16 : 1);
	static constexpr int PS = R * RS;                      // plane stride
	static constexpr size_t SMEM = size_t(WMAX) * PS * 4;
};

template <int LC>
struct RowShape
{
	static constexpr int C = 1 << LC;
	static constexpr int PC = C + C / 32;
	static constexpr size_t SMEM = size_t(WMAX) * PC * 4;
};

constexpr int FS_THREADS = 256;

// Threads per CTA: a shared-memory tile that leaves room for one or two CTAs
// on an SM gets more threads, so that every SM still holds 32 warps.
__host__ __device__ constexpr int col_threads(int lr) { return (lr >= 9) ? 1024 : ((lr == 8) ? 512 : FS_THREADS); }
// A row CTA transforms one plane: 2^(lc-4) radix-16 groups per pass, one per
// thread (at least two warps).
__host__ __device__ constexpr int row_threads(int lc) { return (lc >= 11) ? (1 << (lc - 4)) : 64; }

template <int SET, int LR>
__device__ __forceinline__ void col_fwd_body(const Args &a, const TestDesc &d, uint32_t *sm)
{
	using S = ColShape<LR>;
	constexpr int W = PrimeSet<SET>::W;
	const int n = a.n, lc = n - LR;
	const size_t N = size_t(1) << n, C = size_t(1) << lc;
	const int c0 = blockIdx.x * S::CW;
	const int32_t *src = d.regs + static_cast<size_t>(a.src) * N;
	uint32_t *dst = (a.op == OP_FWD) ? d.zp : d.planes;
	using MP = ColMap<S::RS>;

	if (a.fix)
	{
		// pending carries: digits staged as int32 in the plane-0 area, one
		// thread per 16-digit segment absorbs the incoming carry
		int32_t *dg = reinterpret_cast<int32_t *>(sm);
		for (int e = threadIdx.x; e < S::R * S::CW / 4; e += blockDim.x)
		{
			const int k = e >> (S::CWL - 2), cc = (e & (S::CW / 4 - 1)) * 4;
			const int4 v = *reinterpret_cast<const int4 *>(src + static_cast<size_t>(k) * C + c0 + cc);
			int32_t *p = dg + MP::addr(k, cc);
			p[0] = v.x; p[1] = v.y; p[2] = v.z; p[3] = v.w;
		}
		__syncthreads();
		const size_t nseg = N / SEG;
		int32_t *srcreg = d.regs + static_cast<size_t>(a.src) * N;
		for (int e = threadIdx.x; e < S::R * (S::CW / SEG); e += blockDim.x)
		{
			const int k = e / (S::CW / SEG), sg = e % (S::CW / SEG);
			const size_t j0 = static_cast<size_t>(k) * C + c0 + sg * SEG;
			fix_segment(d, dg + MP::addr(k, sg * SEG), 1, srcreg + j0, take_carry(d, j0 / SEG, nseg, a.op == OP_FWD), a.err);
		}
		__syncthreads();
		for (int e = threadIdx.x; e < S::R * S::CW; e += blockDim.x)
		{
			const int k = e >> S::CWL, cc = e & (S::CW - 1);
			const int i = MP::addr(k, cc);
			const int32_t v = dg[i];
			for_planes<SET>([&](auto PLc) {
				constexpr int PL = decltype(PLc)::value;
				if constexpr (PL > 0) sm[PL * S::PS + i] = ZS<SET, PL>::from_int(v);
			});
			sm[i] = ZS<SET, 0>::from_int(v);
		}
	}
	else
	{
		for (int e = threadIdx.x; e < S::R * S::CW / 4; e += blockDim.x)
		{
			const int k = e >> (S::CWL - 2), cc = (e & (S::CW / 4 - 1)) * 4;
			const int4 v = *reinterpret_cast<const int4 *>(src + static_cast<size_t>(k) * C + c0 + cc);
			for_planes<SET>([&](auto PLc) {
				constexpr int PL = decltype(PLc)::value;
				using Z = ZS<SET, PL>;
				uint32_t *p = sm + PL * S::PS + MP::addr(k, cc);
				p[0] = Z::from_int(v.x); p[1] = Z::from_int(v.y); p[2] = Z::from_int(v.z); p[3] = Z::from_int(v.w);
			});
		}
	}
	__syncthreads();
	run_fwd<SET, LR, false, MP>(sm, S::PS, S::CWL, true, 1u, 0u, a.tab[SET]);
	for (int e = threadIdx.x; e < S::R * S::CW / 4; e += blockDim.x)
	{
		const int k = e >> (S::CWL - 2), cc = (e & (S::CW / 4 - 1)) * 4;
#pragma unroll
		for (int pl = 0; pl < W; ++pl)
		{
			const uint32_t *p = sm + pl * S::PS + MP::addr(k, cc);
			*reinterpret_cast<uint4 *>(dst + pl * N + static_cast<size_t>(k) * C + c0 + cc) = make_uint4(p[0], p[1], p[2], p[3]);
		}
	}
}

// One plane of one row per CTA: blockIdx.x = row * P + plane, P = planes of
// the launch (3, or 4 with packed digits); a CTA whose plane the test does not
// have returns.  The planes of a row are independent until the CRT, so a CTA
// holds one plane (shared memory PC words) and an SM holds as many CTAs as
// its registers allow.
template <int SET, int LC>
__device__ __forceinline__ void row_body(const Args &a, const TestDesc &d, uint32_t *sm)
{
	using S = RowShape<LC>;
	constexpr int W = PrimeSet<SET>::W;
	const int n = a.n, lr = n - LC;
	const size_t N = size_t(1) << n;
	const int P = static_cast<int>(gridDim.x >> lr);
	const int k = static_cast<int>(blockIdx.x) / P, pl = static_cast<int>(blockIdx.x) % P;
	if (pl >= W) return;
	uint32_t *buf = ((a.op == OP_FWD) ? d.zp : d.planes) + static_cast<size_t>(k) * S::C;
	const uint32_t base = a.twist ? 1u : (1u << lr) + static_cast<uint32_t>(k);
	using MP = RowMap<LC>;

	if (a.op != OP_FWD)
	{
		row_core_global<SET, LC, MP>(sm, S::PC, base, a.tab[SET], d.zp + static_cast<size_t>(k) * S::C, N, a.op, buf, N,
									 pl, pl + 1);
		return;
	}
	for (int e = threadIdx.x; e < S::C / 4; e += blockDim.x)
	{
		const uint4 u = *reinterpret_cast<const uint4 *>(buf + pl * N + 4 * e);
		uint32_t *p = sm + MP::addr(4 * e, 0);
		p[0] = u.x; p[1] = u.y; p[2] = u.z; p[3] = u.w;
	}
	__syncthreads();
	run_fwd<SET, LC, false, MP>(sm, S::PC, 0, false, base, 1u, a.tab[SET], pl, pl + 1);
	for (int e = threadIdx.x; e < S::C / 4; e += blockDim.x)
	{
		const uint32_t *p = sm + MP::addr(4 * e, 0);
		*reinterpret_cast<uint4 *>(buf + pl * N + 4 * e) = make_uint4(p[0], p[1], p[2], p[3]);
	}
}

template <int SET, int LR>
__device__ __forceinline__ void col_inv_body(const Args &a, const TestDesc &d, bool dup, uint32_t *sm)
{
	using S = ColShape<LR>;
	constexpr int W = PrimeSet<SET>::W;
	constexpr int SPR = S::CW / SEG;      // segments per tile row
	const int n = a.n, lc = n - LR;
	const size_t N = size_t(1) << n, C = size_t(1) << lc;
	const int c0 = blockIdx.x * S::CW;
	using MP = ColMap<S::RS>;

	for (int e = threadIdx.x; e < S::R * S::CW / 4; e += blockDim.x)
	{
		const int k = e >> (S::CWL - 2), cc = (e & (S::CW / 4 - 1)) * 4;
#pragma unroll
		for (int pl = 0; pl < W; ++pl)
		{
			const uint4 u = *reinterpret_cast<const uint4 *>(d.planes + pl * N + static_cast<size_t>(k) * C + c0 + cc);
			uint32_t *p = sm + pl * S::PS + MP::addr(k, cc);
			p[0] = u.x; p[1] = u.y; p[2] = u.z; p[3] = u.w;
		}
	}
	__syncthreads();
	run_inv<SET, LR, false, MP>(sm, S::PS, S::CWL, true, 1u, 0u, a.tab[SET]);

	int32_t *out = d.regs + static_cast<size_t>(a.dst) * N;
	for (int e = threadIdx.x; e < S::R * SPR; e += blockDim.x)
	{
		const int k = e / SPR, s = e % SPR;
		const size_t j0 = static_cast<size_t>(k) * C + c0 + s * SEG;
		int64_t c = 0;
		int32_t dg[SEG];
#pragma unroll
		for (int i = 0; i < SEG; ++i)
		{
			uint32_t x[3];
#pragma unroll
			for (int pl = 0; pl < W; ++pl) x[pl] = sm[pl * S::PS + MP::addr(k, s * SEG + i)];
			dg[i] = crt_carry<SET>(x, dup ? 1 : 0, d.ck, c);
		}
		int4 *o = reinterpret_cast<int4 *>(out + j0);
#pragma unroll
		for (int i = 0; i < SEG / 4; ++i) o[i] = make_int4(dg[4 * i], dg[4 * i + 1], dg[4 * i + 2], dg[4 * i + 3]);
		d.carry[j0 / SEG] = c;
	}
}

// Columns: tile of CW columns x R rows; first log2 R forward stages.
template <int LR>
__global__ void __launch_bounds__(col_threads(LR)) k_col_fwd(const Args a)
{
	pdl_wait();
	extern __shared__ __align__(16) uint32_t sm[];
	const int t = a.tests[blockIdx.y];
	const TestDesc &d = a.desc[t];
	bool active;
	(void)get_dup(a, d, t, a.j, active);
	if (!active) return;
	if (d.set == 0) col_fwd_body<0, LR>(a, d, sm); else col_fwd_body<1, LR>(a, d, sm);
}

// Rows: the last log2 C forward stages, pointwise, first inverse stages.
template <int LC>
__global__ void __launch_bounds__(row_threads(LC)) k_row(const Args a)
{
	pdl_wait();
	extern __shared__ __align__(16) uint32_t sm[];
	const int t = a.tests[blockIdx.y];
	const TestDesc &d = a.desc[t];
	bool active;
	(void)get_dup(a, d, t, a.j, active);
	if (!active) return;
	if (d.set == 0) row_body<0, LC>(a, d, sm);
	else if (d.set == 1) row_body<1, LC>(a, d, sm);
	else row_body<2, LC>(a, d, sm);
}

// Rows of packed-digit batches (every test on prime set 2), two tests per CTA:
// blockIdx.x = row * 4 + plane, blockIdx.y = pair of the launch's tests.  The
// tests' rows share their roots, which a thread loads once per group for
// both, and the two tests' butterflies are independent chains.  Squarings and
// products only (the forward transform of a multiplicand runs k_row).  A pair
// with one test left (the other one past its exponent, or an odd count) runs
// that test on both lanes and writes it once.
// Four CTAs per SM at 64 registers (16 bytes spilled) for rows of at most
// 4096 points: with the 8-row columns at five, the n = 16 batch 90.1 -> 89.0 us
// per squaring, 16 tests at n = 17 57.5 -> 57.0, against three at 80.
__host__ __device__ constexpr int row2_min_blocks(int lc) { return (row_threads(lc) >= 512) ? 1 : 4; }

template <int LC>
__global__ void __launch_bounds__(row_threads(LC), row2_min_blocks(LC)) k_row2(const Args a, int ntests)
{
	pdl_wait();
	extern __shared__ __align__(16) uint32_t sm[];
	using S = RowShape<LC>;
	const int i0 = 2 * static_cast<int>(blockIdx.y), i1 = i0 + 1;
	int t0 = a.tests[i0], t1 = (i1 < ntests) ? a.tests[i1] : -1;
	bool act0, act1 = (t1 >= 0);
	(void)get_dup(a, a.desc[t0], t0, a.j, act0);
	if (act1) (void)get_dup(a, a.desc[t1], t1, a.j, act1);
	if (!act0 && !act1) return;
	if (!act0) { t0 = t1; act1 = false; }
	const bool store1 = act1;
	if (!act1) t1 = t0;
	const TestDesc &d0 = a.desc[t0], &d1 = a.desc[t1];
	const int n = a.n, lr = n - LC;
	const size_t N = size_t(1) << n;
	const int k = static_cast<int>(blockIdx.x) >> 2, pl = static_cast<int>(blockIdx.x) & 3;
	const size_t off = static_cast<size_t>(pl) * N + static_cast<size_t>(k) * S::C;
	row_core_pair<2, LC, RowMap<LC>>(sm, sm + S::PC, a.twist ? 1u : (1u << lr) + static_cast<uint32_t>(k), a.tab[2],
									 d0.zp + off, d1.zp + off, a.op, d0.planes + off, d1.planes + off, pl, store1);
}

// Rows of a twisted packed launch, two rows of one test per CTA: with the
// six-step twist every row transforms with the roots of base 1, so the pair
// shares each group's roots and runs two independent butterfly chains, as
// k_row2 does for two tests.  blockIdx.x = row pair * 4 + plane, blockIdx.y =
// the launch's test.  Squarings and products only.
template <int LC>
__global__ void __launch_bounds__(row_threads(LC), row2_min_blocks(LC)) k_rowp(const Args a)
{
	pdl_wait();
	extern __shared__ __align__(16) uint32_t sm[];
	using S = RowShape<LC>;
	const int t = a.tests[blockIdx.y];
	const TestDesc &d = a.desc[t];
	bool active;
	(void)get_dup(a, d, t, a.j, active);
	if (!active) return;
	const size_t N = size_t(1) << a.n;
	const int k = 2 * (static_cast<int>(blockIdx.x) >> 2), pl = static_cast<int>(blockIdx.x) & 3;
	const size_t off = static_cast<size_t>(pl) * N + static_cast<size_t>(k) * S::C;
	row_core_pair<2, LC, RowMap<LC>>(sm, sm + S::PC, 1u, a.tab[2], d.zp + off, d.zp + off + S::C, a.op,
									 d.planes + off, d.planes + off + S::C, pl, true);
}

// Columns: last log2 R inverse stages, CRT, carry inside 16-digit segments.
template <int LR>
__global__ void __launch_bounds__(col_threads(LR)) k_col_inv(const Args a)
{
	pdl_wait();
	extern __shared__ __align__(16) uint32_t sm[];
	const int t = a.tests[blockIdx.y];
	const TestDesc &d = a.desc[t];
	bool active;
	const bool dup = get_dup(a, d, t, a.j, active);
	if (!active) return;
	if (d.set == 0) col_inv_body<0, LR>(a, d, dup, sm); else col_inv_body<1, LR>(a, d, dup, sm);
}

// ---- transforms of one thread's registers.
//
// A whole 2^L-point transform (base `base`, stages 0 .. L-1 of it) on an
// array the thread owns, in the passes of Sched<L>: pass p covers the stages
// 4p .. 4p + r - 1 as groups of 2^r elements with stride 2^sh, sh = L - 4p - r;
// the groups of sub-block blk share the roots tw[(((base << 4p) + blk) << t) + sb],
// loaded once per sub-block.  The same butterflies in the same order as
// pass_all over a tile, so the results are identical.  base >= 2 (no
// normalisation: never the first stage of a whole transform).
template <class Z, int L>
__device__ __forceinline__ void fwd_thread(const Z &z, uint32_t (&x)[1 << L], uint32_t base, const uint32_t *__restrict__ tw)
{
	if constexpr (L <= 4) { fwd_reg<Z, L>(z, x, base, tw); return; }
	static_for<0, Sched<L>::NP>([&](auto P) {
		constexpr int p = decltype(P)::value, s0 = 4 * p, r = Sched<L>::r(p), sh = L - s0 - r;
#pragma unroll
		for (int blk = 0; blk < (1 << s0); ++blk)
		{
			typename Z::root_t w[(1 << r) - 1];
			load_twiddles<r>(w, (base << s0) + static_cast<uint32_t>(blk), tw);
#pragma unroll
			for (int t = 0; t < r; ++t)
			{
				const int half = 1 << (r - 1 - t);
#pragma unroll
				for (int sb = 0; sb < (1 << t); ++sb)
#pragma unroll
					for (int mm = 0; mm < half; ++mm)
#pragma unroll
						for (int o = 0; o < (1 << sh); ++o)
						{
							const int i0 = (blk << (L - s0)) + o + ((sb * 2 * half + mm) << sh);
							bfly_ct(z, x[i0], x[i0 + (half << sh)], w[(1 << t) - 1 + sb]);
						}
			}
		}
	});
}

template <class Z, int L>
__device__ __forceinline__ void inv_thread(const Z &z, uint32_t (&x)[1 << L], uint32_t base, const uint32_t *__restrict__ twi)
{
	if constexpr (L <= 4) { inv_reg<Z, L>(z, x, base, twi, false, 0u, 0u); return; }
	constexpr int NP = Sched<L>::NP;
	static_for<0, NP>([&](auto Q) {
		constexpr int p = NP - 1 - decltype(Q)::value, s0 = 4 * p, r = Sched<L>::r(p), sh = L - s0 - r;
#pragma unroll
		for (int blk = 0; blk < (1 << s0); ++blk)
		{
			typename Z::root_t w[(1 << r) - 1];
			load_twiddles<r>(w, (base << s0) + static_cast<uint32_t>(blk), twi);
#pragma unroll
			for (int t = r - 1; t >= 0; --t)
			{
				const int half = 1 << (r - 1 - t);
#pragma unroll
				for (int sb = 0; sb < (1 << t); ++sb)
#pragma unroll
					for (int mm = 0; mm < half; ++mm)
#pragma unroll
						for (int o = 0; o < (1 << sh); ++o)
						{
							const int i0 = (blk << (L - s0)) + o + ((sb * 2 * half + mm) << sh);
							bfly_gs(z, x[i0], x[i0 + (half << sh)], w[(1 << t) - 1 + sb]);
						}
			}
		}
	});
}

// ---- six-step middle pass.
//
// With R = R1 R2 rows (R1 = 2^MID_LR1), the column transform of length R is
// split: the R1-point column pass (stages 0 .. MID_LR1-1) is the four-step
// column kernel of R1 rows over the same N, and this pass runs stages
// MID_LR1 .. MID_LR1 + LR2 - 1: for block m < R1, rows m R2 .. m R2 + R2 - 1
// of the R x C matrix hold 2^LR2-point transforms down each column with base
// R1 + m.  Tile: R2 rows x CW columns of every plane, planes in and out.
constexpr int MID_LR1 = 4;

// The six-step twist.  Row k of the R x C matrix the middle pass leaves
// (R = 2^lr, element c of row k at k C + c) is the block of the negacyclic
// transform at table base R + k.  Its evaluation points are nu_k times those
// of the length-C transform at base 1, nu_k = psi^(2 brev_lr(k) + 1 - R), so
// its forward transform is the base-1 transform of the row with element c
// multiplied by nu_k^c, and its inverse is the base-1 inverse followed by
// nu_k^-c.  With the twist in the middle pass every row reads the same C - 1
// roots (entries 1 .. C-1 of the table, psi^(R brev(e)) = the roots of the
// length-C transform) instead of its own.  With k = m 2^LR2 + q (m the
// middle block, q the register):
//     nu_k^c = H[m][c] G[c]^brev_LR2(q),
//     H[m][c] = psi^(c (2 brev_4(m) + 1 - R)),  G[c] = psi^(32 c).
// Table of one prime and direction (k_twist; psi^-1 for the inverse): H as
// 16 C words in Montgomery form, then G as C root entries.  (The 64-row
// pair pass, k_midp, does not twist: at its register limit the twist cost
// more than the rows gained.)
__host__ __device__ constexpr int brev_c(int j, int bits)
{
	int r = 0;
	for (int i = 0; i < bits; ++i) r |= ((j >> i) & 1) << (bits - 1 - i);
	return r;
}

__device__ __forceinline__ void load_root(RootS &r, const uint32_t *t, size_t i)
{
	const uint2 u = __ldg(reinterpret_cast<const uint2 *>(t) + i);
	r = RootS{ u.x, u.y };
}

__device__ __forceinline__ void load_root(RootM &r, const uint32_t *t, size_t i) { r = RootM{ __ldg(t + i) }; }

// x[i] times f g^brev_LB(i) for i < 2^LB (f in Montgomery form, g a root entry).
template <class Z, int LB>
__device__ __forceinline__ void twist_regs(const Z &z, uint32_t (&x)[1 << LB], uint32_t f, typename Z::root_t g)
{
#pragma unroll
	for (int j = 0; j < (1 << LB); ++j)
	{
		const int i = brev_c(j, LB);
		x[i] = z.mul(x[i], f);
		if (j + 1 < (1 << LB)) f = z.mulr(f, g);
	}
}

// H[m][c] and G[c] of a twist table with C columns.
__device__ __forceinline__ uint32_t twist_start(const uint32_t *tt, int m, size_t c, size_t C)
{
	return __ldg(tt + static_cast<size_t>(m) * C + c);
}

template <class Z>
__device__ __forceinline__ typename Z::root_t twist_step(const uint32_t *tt, size_t c, size_t C)
{
	typename Z::root_t g;
	load_root(g, tt + 16 * C, c);
	return g;
}

// Unpadded column tile of the middle pass (no CRT reads it): a warp's 32
// consecutive columns of one row are 32 consecutive words, and the 16-byte
// staging writes of 8 consecutive threads cover whole rows.
template <int RS>
struct ColMapU
{
	__device__ __forceinline__ static int addr(int i, int lane) { return i * RS + lane; }
	__host__ __device__ static constexpr int off(int m, int step) { return m * step * RS; }
};

template <int LR2>
struct MidShape
{
	static constexpr int R = 1 << LR2;
	static constexpr int CW = col_width(LR2);
	static constexpr int CWL = ilog2c(CW);
	static constexpr int PS = R * CW;                      // plane stride
	static constexpr size_t SMEM = size_t(4) * PS * 4;     // up to four planes
};

template <int SET, int LR2, bool INV>
__device__ __forceinline__ void mid_body(const Args &a, const TestDesc &d, uint32_t *sm)
{
	using S = MidShape<LR2>;
	constexpr int W = PrimeSet<SET>::W;
	const int lr = MID_LR1 + LR2, lc = a.n - lr;
	const size_t N = size_t(1) << a.n, C = size_t(1) << lc;
	const int tiles = static_cast<int>(C / S::CW);
	const int m = blockIdx.x / tiles;                      // block of R2 rows
	const size_t c0 = static_cast<size_t>(blockIdx.x % tiles) * S::CW;
	const size_t row0 = static_cast<size_t>(m) << LR2;
	// the forward transform of a multiplicand (OP_FWD) lives in zp
	uint32_t *planes = ((a.op == OP_FWD) ? d.zp : d.planes) + row0 * C + c0;
	using MP = ColMapU<S::CW>;
	for (int e = threadIdx.x; e < S::R * S::CW / 4; e += blockDim.x)
	{
		const int k = e >> (S::CWL - 2), cc = (e & (S::CW / 4 - 1)) * 4;
#pragma unroll
		for (int pl = 0; pl < W; ++pl)
			*reinterpret_cast<uint4 *>(sm + pl * S::PS + MP::addr(k, cc)) =
				*reinterpret_cast<const uint4 *>(planes + pl * N + static_cast<size_t>(k) * C + cc);
	}
	__syncthreads();
	const uint32_t base = (1u << MID_LR1) + static_cast<uint32_t>(m);
	if constexpr (INV) run_inv<SET, LR2, false, MP>(sm, S::PS, S::CWL, true, base, 0u, a.tab[SET]);
	else run_fwd<SET, LR2, false, MP>(sm, S::PS, S::CWL, true, base, 0u, a.tab[SET]);
	for (int e = threadIdx.x; e < S::R * S::CW / 4; e += blockDim.x)
	{
		const int k = e >> (S::CWL - 2), cc = (e & (S::CW / 4 - 1)) * 4;
#pragma unroll
		for (int pl = 0; pl < W; ++pl)
			*reinterpret_cast<uint4 *>(planes + pl * N + static_cast<size_t>(k) * C + cc) =
				*reinterpret_cast<const uint4 *>(sm + pl * S::PS + MP::addr(k, cc));
	}
}

template <int LR2, bool INV>
__global__ void __launch_bounds__(col_threads(LR2)) k_mid(const Args a)
{
	pdl_wait();
	extern __shared__ __align__(16) uint32_t sm[];
	const int t = a.tests[blockIdx.y];
	const TestDesc &d = a.desc[t];
	bool active;
	(void)get_dup(a, d, t, a.j, active);
	if (!active) return;
	if (d.set == 0) mid_body<0, LR2, INV>(a, d, sm);
	else if (d.set == 1) mid_body<1, LR2, INV>(a, d, sm);
	else mid_body<2, LR2, INV>(a, d, sm);
}

// The middle pass in registers: a thread owns one column of one plane of one
// block of 2^LR2 rows (2^LR2 words at stride C, a warp's 32 consecutive columns
// making each load and store one 128-byte line), so the pass needs no shared
// memory and no barrier.  blockIdx.x = (m P + plane) (C / MIDR_THREADS) + chunk
// of MIDR_THREADS columns, P = planes of the launch; a CTA whose plane the test
// does not have returns.
constexpr int MIDR_THREADS = 128;
constexpr int MIDR_LOG = 7;

template <int SET, int LR2, bool INV>
__device__ __forceinline__ void midr_body(const Args &a, const TestDesc &d, int m, int pl, size_t c)
{
	if (pl >= PrimeSet<SET>::W) return;
	const int lc = a.n - MID_LR1 - LR2;
	const size_t N = size_t(1) << a.n, C = size_t(1) << lc;
	uint32_t *p = ((a.op == OP_FWD) ? d.zp : d.planes) + static_cast<size_t>(pl) * N +
				  ((static_cast<size_t>(m) << LR2) << lc) + c;
	const auto z = prime_rt<SET>(pl);
	using Z = decltype(z);
	uint32_t x[1 << LR2];
#pragma unroll
	for (int k = 0; k < (1 << LR2); ++k) x[k] = p[k * C];
	const uint32_t base = (1u << MID_LR1) + static_cast<uint32_t>(m);
	if constexpr (INV)
	{
		if (a.twist)
		{
			const uint32_t *tt = a.tab[SET].ti[pl];
			twist_regs<Z, LR2>(z, x, twist_start(tt, m, c, C), twist_step<Z>(tt, c, C));
		}
		inv_thread<Z, LR2>(z, x, base, a.tab[SET].iv[pl]);
	}
	else
	{
		fwd_thread<Z, LR2>(z, x, base, a.tab[SET].fw[pl]);
		if (a.twist)
		{
			const uint32_t *tt = a.tab[SET].tf[pl];
			twist_regs<Z, LR2>(z, x, twist_start(tt, m, c, C), twist_step<Z>(tt, c, C));
		}
	}
#pragma unroll
	for (int k = 0; k < (1 << LR2); ++k) p[k * C] = x[k];
}

// 32-word columns (lr2 = 5) fit four CTAs per SM in 128 registers.
__host__ __device__ constexpr int midr_min_blocks(int lr2) { return (lr2 == 5) ? 4 : 1; }

template <int LR2, bool INV>
__global__ void __launch_bounds__(MIDR_THREADS, midr_min_blocks(LR2)) k_midr(const Args a)
{
	pdl_wait();
	const int t = a.tests[blockIdx.y];
	const TestDesc &d = a.desc[t];
	bool active;
	(void)get_dup(a, d, t, a.j, active);
	if (!active) return;
	const int chunks_log = a.n - MID_LR1 - LR2 - MIDR_LOG;
	const int P = static_cast<int>(gridDim.x >> (MID_LR1 + chunks_log));
	const int q = static_cast<int>(blockIdx.x >> chunks_log);
	const int m = q / P, pl = q % P;
	const size_t c = (static_cast<size_t>(blockIdx.x & ((1u << chunks_log) - 1)) << MIDR_LOG) + threadIdx.x;
	if (d.set == 0) midr_body<0, LR2, INV>(a, d, m, pl, c);
	else if (d.set == 1) midr_body<1, LR2, INV>(a, d, m, pl, c);
	else midr_body<2, LR2, INV>(a, d, m, pl, c);
}

// The 64-point middle pass (lr2 = 6) on thread pairs: lanes 2c' and 2c' + 1 of a
// warp share column c of one plane of one block, 32 words each, so that a
// thread holds what the 32-point pass holds (four CTAs per SM in 128
// registers) instead of 64 words and their roots.  Forward: half h loads the
// rows 16 h .. 16 h + 15 and 32 + 16 h .. 32 + 16 h + 15, whose first-stage
// butterflies (rows j, j + 32) it then owns, and after that stage swaps 16
// words with its partner so that it holds the rows 32 h .. 32 h + 31, on which
// stages 1 .. 5 are the 32-point transform of base 2 base + h.  Inverse: the
// same steps in reverse order.  The same butterflies with the same roots as
// k_midr<6>, so the results are identical.  blockIdx.x = (m P + plane)
// (C / MIDP_COLS) + chunk of MIDP_COLS columns.
constexpr int MIDP_THREADS = 128;
constexpr int MIDP_COLS = MIDP_THREADS / 2;
constexpr int MIDP_COLS_LOG = 6;

template <int SET, bool INV>
__device__ __forceinline__ void midp_body(const Args &a, const TestDesc &d, int m, int pl, size_t c, int h)
{
	if (pl >= PrimeSet<SET>::W) return;
	constexpr int LR2 = 6;
	const int lc = a.n - MID_LR1 - LR2;
	const size_t N = size_t(1) << a.n, C = size_t(1) << lc;
	uint32_t *p = ((a.op == OP_FWD) ? d.zp : d.planes) + static_cast<size_t>(pl) * N +
				  ((static_cast<size_t>(m) << LR2) << lc) + c;
	const auto z = prime_rt<SET>(pl);
	using Z = decltype(z);
	const uint32_t base = (1u << MID_LR1) + static_cast<uint32_t>(m);
	uint32_t x[32];
	if constexpr (!INV)
	{
#pragma unroll
		for (int i = 0; i < 16; ++i)
		{
			x[i] = p[static_cast<size_t>(16 * h + i) * C];
			x[16 + i] = p[static_cast<size_t>(32 + 16 * h + i) * C];
		}
		typename Z::root_t w0[1];
		load_twiddles<1>(w0, base, a.tab[SET].fw[pl]);
#pragma unroll
		for (int i = 0; i < 16; ++i) bfly_ct(z, x[i], x[16 + i], w0[0]);
		// h = 0 keeps rows 0..15 and takes 16..31; h = 1 keeps 48..63 and takes 32..47
#pragma unroll
		for (int i = 0; i < 16; ++i)
		{
			const uint32_t send = h ? x[i] : x[16 + i];
			const uint32_t recv = __shfl_xor_sync(0xffffffffu, send, 1);
			if (h) x[i] = recv; else x[16 + i] = recv;
		}
		fwd_thread<Z, 5>(z, x, 2u * base + static_cast<uint32_t>(h), a.tab[SET].fw[pl]);
#pragma unroll
		for (int i = 0; i < 32; ++i) p[static_cast<size_t>(32 * h + i) * C] = x[i];
	}
	else
	{
#pragma unroll
		for (int i = 0; i < 32; ++i) x[i] = p[static_cast<size_t>(32 * h + i) * C];
		inv_thread<Z, 5>(z, x, 2u * base + static_cast<uint32_t>(h), a.tab[SET].iv[pl]);
		// back to the pairs of the first stage: h = 0 holds rows 0..15 with
		// 32..47, h = 1 rows 16..31 with 48..63
#pragma unroll
		for (int i = 0; i < 16; ++i)
		{
			const uint32_t send = h ? x[i] : x[16 + i];
			const uint32_t recv = __shfl_xor_sync(0xffffffffu, send, 1);
			if (h) x[i] = recv; else x[16 + i] = recv;
		}
		typename Z::root_t w0[1];
		load_twiddles<1>(w0, base, a.tab[SET].iv[pl]);
#pragma unroll
		for (int i = 0; i < 16; ++i) bfly_gs(z, x[i], x[16 + i], w0[0]);
#pragma unroll
		for (int i = 0; i < 16; ++i)
		{
			p[static_cast<size_t>(16 * h + i) * C] = x[i];
			p[static_cast<size_t>(32 + 16 * h + i) * C] = x[16 + i];
		}
	}
}

template <bool INV>
__global__ void __launch_bounds__(MIDP_THREADS, 4) k_midp(const Args a)
{
	pdl_wait();
	const int t = a.tests[blockIdx.y];
	const TestDesc &d = a.desc[t];
	bool active;
	(void)get_dup(a, d, t, a.j, active);
	if (!active) return;
	const int chunks_log = a.n - MID_LR1 - 6 - MIDP_COLS_LOG;
	const int P = static_cast<int>(gridDim.x >> (MID_LR1 + chunks_log));
	const int q = static_cast<int>(blockIdx.x >> chunks_log);
	const int m = q / P, pl = q % P;
	const int h = static_cast<int>(threadIdx.x & 1);
	const size_t c = (static_cast<size_t>(blockIdx.x & ((1u << chunks_log) - 1)) << MIDP_COLS_LOG) + (threadIdx.x >> 1);
	if (d.set == 0) midp_body<0, INV>(a, d, m, pl, c, h);
	else if (d.set == 1) midp_body<1, INV>(a, d, m, pl, c, h);
	else midp_body<2, INV>(a, d, m, pl, c, h);
}

// ---- four-step with R <= 16 rows: one thread owns a whole column.

constexpr int COLR_THREADS = 256;

template <int SET, int LR>
__device__ __forceinline__ void col_fwd_reg_body(const Args &a, const TestDesc &d, int32_t *sm)
{
	constexpr int R = 1 << LR, T = COLR_THREADS;
	const int n = a.n;
	const size_t N = size_t(1) << n, C = size_t(1) << (n - LR);
	const size_t c0 = static_cast<size_t>(blockIdx.x) * T;
	const int tid = threadIdx.x;
	int32_t *const srcreg = d.regs + static_cast<size_t>(a.src) * N;
	const int32_t *src = srcreg + c0 + tid;
	uint32_t *dst = ((a.op == OP_FWD) ? d.zp : d.planes) + c0 + tid;
	int32_t dv[R];
#pragma unroll
	for (int k = 0; k < R; ++k) dv[k] = src[k * C];
	if (a.fix)
	{
		// pending carries: stage the tile [R][T] (digit c of row k at k RW +
		// c + c / 16, so that the threads' 16-digit segments start in distinct
		// banks), one thread per segment
		constexpr int RW = T + T / SEG;
#pragma unroll
		for (int k = 0; k < R; ++k) sm[k * RW + tid + tid / SEG] = dv[k];
		__syncthreads();
		const size_t nseg = N / SEG;
		for (int e = tid; e < R * (T / SEG); e += T)
		{
			const int k = e / (T / SEG), s = e % (T / SEG);
			const size_t j0 = static_cast<size_t>(k) * C + c0 + s * SEG;
			fix_segment(d, sm + k * RW + s * (SEG + 1), 1, srcreg + j0, take_carry(d, j0 / SEG, nseg, a.op == OP_FWD),
						a.err);
		}
		__syncthreads();
#pragma unroll
		for (int k = 0; k < R; ++k) dv[k] = sm[k * RW + tid + tid / SEG];
	}
	for_planes<SET>([&](auto PLc) {
		constexpr int PL = decltype(PLc)::value;
		using Z = ZS<SET, PL>;
		uint32_t x[R];
#pragma unroll
		for (int k = 0; k < R; ++k) x[k] = Z::from_int(dv[k]);
		fwd_reg<Z, LR>(Z{}, x, 1u, a.tab[SET].fw[PL]);
#pragma unroll
		for (int k = 0; k < R; ++k) dst[PL * N + k * C] = x[k];
	});
}

// Inverse column transform in registers, then the tile (R rows x 256
// columns) goes through shared memory so that each thread takes one 16-digit
// row segment for CRT and carry.
template <int SET, int LR>
__device__ __forceinline__ void col_inv_reg_body(const Args &a, const TestDesc &d, bool dup, uint32_t *sm)
{
	constexpr int R = 1 << LR, W = PrimeSet<SET>::W;
	constexpr int T = COLR_THREADS, RS = T + T / 16, PS = R * RS, SPR = T / SEG;
	const int n = a.n;
	const size_t N = size_t(1) << n, C = size_t(1) << (n - LR);
	const size_t c0 = static_cast<size_t>(blockIdx.x) * T;
	const int tid = threadIdx.x;
	using MP = ColMap<RS>;
	for_planes<SET>([&](auto PLc) {
		constexpr int PL = decltype(PLc)::value;
		using Z = ZS<SET, PL>;
		const uint32_t *src = d.planes + PL * N + c0 + tid;
		uint32_t x[R];
#pragma unroll
		for (int k = 0; k < R; ++k) x[k] = src[k * C];
		inv_reg<Z, LR>(Z{}, x, 1u, a.tab[SET].iv[PL], true, __ldg(&a.tab[SET].fw[PL][0]), __ldg(&a.tab[SET].iv[PL][0]));
#pragma unroll
		for (int k = 0; k < R; ++k) sm[PL * PS + MP::addr(k, tid)] = x[k];
	});
	__syncthreads();
	int32_t *out = d.regs + static_cast<size_t>(a.dst) * N;
	for (int e = tid; e < R * SPR; e += T)
	{
		const int k = e / SPR, s = e % SPR;
		const size_t j0 = static_cast<size_t>(k) * C + c0 + s * SEG;
		int64_t cr = 0;
		int32_t dg[SEG];
#pragma unroll
		for (int i = 0; i < SEG; ++i)
		{
			uint32_t x[3];
#pragma unroll
			for (int pl = 0; pl < W; ++pl) x[pl] = sm[pl * PS + MP::addr(k, s * SEG + i)];
			dg[i] = crt_carry<SET>(x, dup ? 1 : 0, d.ck, cr);
		}
		int4 *o = reinterpret_cast<int4 *>(out + j0);
#pragma unroll
		for (int i = 0; i < SEG / 4; ++i) o[i] = make_int4(dg[4 * i], dg[4 * i + 1], dg[4 * i + 2], dg[4 * i + 3]);
		d.carry[j0 / SEG] = cr;
	}
}

// Shared memory: [R][T + T/16] int32 staging of the digits when fixing carries.
template <int LR>
__global__ void __launch_bounds__(COLR_THREADS) k_colr_fwd(const Args a)
{
	pdl_wait();
	__shared__ int32_t sm[(1 << LR) * (COLR_THREADS + COLR_THREADS / SEG)];
	const int t = a.tests[blockIdx.y];
	const TestDesc &d = a.desc[t];
	bool active;
	(void)get_dup(a, d, t, a.j, active);
	if (!active) return;
	if (d.set == 0) col_fwd_reg_body<0, LR>(a, d, sm); else col_fwd_reg_body<1, LR>(a, d, sm);
}

template <int LR>
struct ColRegShape
{
	static constexpr size_t SMEM = size_t(WMAX) * (1 << LR) * (COLR_THREADS + COLR_THREADS / 16) * 4;
};

template <int LR>
__global__ void __launch_bounds__(COLR_THREADS) k_colr_inv(const Args a)
{
	pdl_wait();
	extern __shared__ __align__(16) uint32_t sm[];
	const int t = a.tests[blockIdx.y];
	const TestDesc &d = a.desc[t];
	bool active;
	const bool dup = get_dup(a, d, t, a.j, active);
	if (!active) return;
	if (d.set == 0) col_inv_reg_body<0, LR>(a, d, dup, sm); else col_inv_reg_body<1, LR>(a, d, dup, sm);
}

// ---- plane-split register columns, for batches too small to fill the GPU
// with one thread per column: a CTA takes CS_T columns and has a thread per
// (plane, column), WMAX planes (threads of planes the test does not have only
// join the barriers).  Same arithmetic in the same order as the kernels above.

constexpr int CS_T = 64;

template <int SET, int LR>
__device__ __forceinline__ void col_fwd_split_body(const Args &a, const TestDesc &d, int32_t *sm)
{
	constexpr int R = 1 << LR, T = CS_T, NT = WMAX * T, RW = T + T / SEG;
	const size_t N = size_t(1) << a.n, C = size_t(1) << (a.n - LR);
	const size_t c0 = static_cast<size_t>(blockIdx.x) * T;
	const int tid = threadIdx.x, c = tid % T, pl = tid / T;
	int32_t *const srcreg = d.regs + static_cast<size_t>(a.src) * N;
	if (a.fix)
	{
		// the tile [R][T], digit c of row k at k RW + c + c / 16; one thread per segment
		for (int e = tid; e < R * T; e += NT)
		{
			const int k = e / T, cc = e % T;
			sm[k * RW + cc + cc / SEG] = srcreg[static_cast<size_t>(k) * C + c0 + cc];
		}
		__syncthreads();
		const size_t nseg = N / SEG;
		for (int e = tid; e < R * (T / SEG); e += NT)
		{
			const int k = e / (T / SEG), s = e % (T / SEG);
			const size_t j0 = static_cast<size_t>(k) * C + c0 + s * SEG;
			fix_segment(d, sm + k * RW + s * (SEG + 1), 1, srcreg + j0, take_carry(d, j0 / SEG, nseg, a.op == OP_FWD),
						a.err);
		}
		__syncthreads();
	}
	if (pl >= PrimeSet<SET>::W) return;
	const auto z = prime_rt<SET>(pl);
	uint32_t x[R];
#pragma unroll
	for (int k = 0; k < R; ++k)
		x[k] = z.from_int(a.fix ? sm[k * RW + c + c / SEG] : srcreg[static_cast<size_t>(k) * C + c0 + c]);
	fwd_reg<decltype(z), LR>(z, x, 1u, a.tab[SET].fw[pl]);
	uint32_t *dst = ((a.op == OP_FWD) ? d.zp : d.planes) + pl * N + c0 + c;
#pragma unroll
	for (int k = 0; k < R; ++k) dst[k * C] = x[k];
}

template <int SET, int LR>
__device__ __forceinline__ void col_inv_split_body(const Args &a, const TestDesc &d, bool dup, uint32_t *sm)
{
	constexpr int R = 1 << LR, W = PrimeSet<SET>::W;
	constexpr int T = CS_T, NT = WMAX * T, RS = T + T / 16, PS = R * RS, SPR = T / SEG;
	const size_t N = size_t(1) << a.n, C = size_t(1) << (a.n - LR);
	const size_t c0 = static_cast<size_t>(blockIdx.x) * T;
	const int tid = threadIdx.x, c = tid % T, pl = tid / T;
	using MP = ColMap<RS>;
	if (pl < W)
	{
		const auto z = prime_rt<SET>(pl);
		const uint32_t *src = d.planes + pl * N + c0 + c;
		uint32_t x[R];
#pragma unroll
		for (int k = 0; k < R; ++k) x[k] = src[k * C];
		inv_reg<decltype(z), LR>(z, x, 1u, a.tab[SET].iv[pl], true, __ldg(&a.tab[SET].fw[pl][0]),
								 __ldg(&a.tab[SET].iv[pl][0]));
#pragma unroll
		for (int k = 0; k < R; ++k) sm[pl * PS + MP::addr(k, c)] = x[k];
	}
	__syncthreads();
	int32_t *out = d.regs + static_cast<size_t>(a.dst) * N;
	for (int e = tid; e < R * SPR; e += NT)
	{
		const int k = e / SPR, s = e % SPR;
		const size_t j0 = static_cast<size_t>(k) * C + c0 + s * SEG;
		int64_t cr = 0;
		int32_t dg[SEG];
#pragma unroll
		for (int i = 0; i < SEG; ++i)
		{
			uint32_t x[3];
#pragma unroll
			for (int q = 0; q < W; ++q) x[q] = sm[q * PS + MP::addr(k, s * SEG + i)];
			dg[i] = crt_carry<SET>(x, dup ? 1 : 0, d.ck, cr);
		}
		int4 *o = reinterpret_cast<int4 *>(out + j0);
#pragma unroll
		for (int i = 0; i < SEG / 4; ++i) o[i] = make_int4(dg[4 * i], dg[4 * i + 1], dg[4 * i + 2], dg[4 * i + 3]);
		d.carry[j0 / SEG] = cr;
	}
}

template <int LR>
__global__ void __launch_bounds__(WMAX * CS_T) k_colr_fwd_s(const Args a)
{
	pdl_wait();
	__shared__ int32_t sm[(1 << LR) * (CS_T + CS_T / SEG)];
	const int t = a.tests[blockIdx.y];
	const TestDesc &d = a.desc[t];
	bool active;
	(void)get_dup(a, d, t, a.j, active);
	if (!active) return;
	if (d.set == 0) col_fwd_split_body<0, LR>(a, d, sm); else col_fwd_split_body<1, LR>(a, d, sm);
}

template <int LR>
__global__ void __launch_bounds__(WMAX * CS_T) k_colr_inv_s(const Args a)
{
	pdl_wait();
	__shared__ __align__(16) uint32_t sm[WMAX * (1 << LR) * (CS_T + CS_T / 16)];
	const int t = a.tests[blockIdx.y];
	const TestDesc &d = a.desc[t];
	bool active;
	const bool dup = get_dup(a, d, t, a.j, active);
	if (!active) return;
	if (d.set == 0) col_inv_split_body<0, LR>(a, d, dup, sm); else col_inv_split_body<1, LR>(a, d, dup, sm);
}

// ---- packed digits (prime set 2).
//
// Coefficient i of the packed transform (N' = N/2 points, a.n = n - 1 in these
// launches) is D_i = d_2i + b d_2i+1.  A 16-digit carry segment is 8
// coefficients; its carry is PK_CARRY values (d.carry[PK_CARRY s + k]).
// Register column kernels (R = 2^LR <= 16 rows, a thread per packed column);
// the rows are k_row with prime set 2.

constexpr int PCOL_THREADS = 256;

// The word of root-table entry 0 that holds the normalisation of a packed
// column size: 1 (for inputs D 2^-32) with 8-row columns, 0 with 16-row ones.
__host__ __device__ constexpr int pcol_norm_word(int lr) { return (lr == 3) ? 1 : 0; }

// Takes (and clears) the packed carry into segment s: the previous
// segment's, negated across the wrap (b^N = -1).
__device__ __forceinline__ void take_carry5(const TestDesc &d, size_t s, size_t nseg, int64_t (&c)[PK_CARRY],
											bool clear = true)
{
	const size_t src = (s == 0) ? nseg - 1 : s - 1;
	int64_t *const p = d.carry + PK_CARRY * src;
#pragma unroll
	for (int k = 0; k < PK_CARRY; ++k)
	{
		const int64_t v = p[k];
		if (clear && (v != 0)) p[k] = 0;
		c[k] = (s == 0) ? -v : v;
	}
}

__device__ __forceinline__ void fix_segment5(const TestDesc &d, int32_t *seg, int32_t *g, size_t s, size_t nseg,
											 bool clear, uint32_t *err)
{
	int64_t c[PK_CARRY];
	take_carry5(d, s, nseg, c, clear);
	bool any = false;
#pragma unroll
	for (int k = 0; k < PK_CARRY; ++k) any |= (c[k] != 0);
	if (!any) return;
	int32_t dg[SEG], old[SEG];
#pragma unroll
	for (int i = 0; i < SEG; ++i) old[i] = dg[i] = seg[i];
	if (!absorb5<SEG>(dg, c, d.ck)) atomicOr(err, 1u);
#pragma unroll
	for (int i = 0; i < SEG; ++i)
		if (dg[i] != old[i]) { seg[i] = dg[i]; g[i] = dg[i]; }     // write back the digits that changed
}

// Digits -> packed residues -> first LR forward stages (one packed column per
// thread); absorbs pending packed carries of register src first.
template <int LR>
__device__ __forceinline__ void pcol_fwd_body(const Args &a, const TestDesc &d, int32_t *sm)
{
	constexpr int R = 1 << LR, T = PCOL_THREADS, RW = 2 * T + 2 * T / SEG;
	const size_t Np = size_t(1) << a.n, Cp = size_t(1) << (a.n - LR);
	const size_t c0 = static_cast<size_t>(blockIdx.x) * T;
	const int tid = threadIdx.x;
	int32_t *const srcreg = d.regs + static_cast<size_t>(a.src) * (2 * Np);
	uint32_t *dst = ((a.op == OP_FWD) ? d.zp : d.planes) + c0 + tid;
	int32_t d0[R], d1[R];
#pragma unroll
	for (int k = 0; k < R; ++k)
	{
		const int2 v = *reinterpret_cast<const int2 *>(srcreg + 2 * (static_cast<size_t>(k) * Cp + c0 + tid));
		d0[k] = v.x; d1[k] = v.y;
	}
	if (a.fix)
	{
		// digit j of row k at k RW + j + j / 16: the threads' 16-digit segments
		// start in distinct banks
		const int o = 2 * tid + tid / (SEG / 2);
#pragma unroll
		for (int k = 0; k < R; ++k) { sm[k * RW + o] = d0[k]; sm[k * RW + o + 1] = d1[k]; }
		__syncthreads();
		const size_t nseg = (2 * Np) / SEG;
		for (int e = tid; e < R * (2 * T / SEG); e += T)
		{
			const int k = e / (2 * T / SEG), s = e % (2 * T / SEG);
			const size_t j0 = 2 * (static_cast<size_t>(k) * Cp + c0) + static_cast<size_t>(s) * SEG;
			fix_segment5(d, sm + k * RW + s * (SEG + 1), srcreg + j0, j0 / SEG, nseg, a.op == OP_FWD, a.err);
		}
		__syncthreads();
#pragma unroll
		for (int k = 0; k < R; ++k) { d0[k] = sm[k * RW + o]; d1[k] = sm[k * RW + o + 1]; }
	}
	// 8-row columns pack as D 2^-32 (pack_residue), 16-row ones as D
	const uint32_t bb = d.b;
	for_planes<2>([&](auto PLc) {
		constexpr int PL = decltype(PLc)::value;
		using Z = ZS<2, PL>;
		uint32_t x[R];
		if constexpr (LR == 3)
		{
#pragma unroll
			for (int k = 0; k < R; ++k) x[k] = pack_residue(Z{}, pack_value(d0[k], d1[k], bb));
		}
		else
		{
			const uint32_t bm = d.pk.bm[PL];
#pragma unroll
			for (int k = 0; k < R; ++k) x[k] = Z::add(Z::from_int(d0[k]), Z::mul(Z::from_int(d1[k]), bm));
		}
		fwd_reg<Z, LR>(Z{}, x, 1u, a.tab[2].fw[PL]);
#pragma unroll
		for (int k = 0; k < R; ++k) dst[PL * Np + k * Cp] = x[k];
	});
}

// Tile of the packed inverse column kernel: coefficient c of row k at
// k RS + (c % 8) Q + c / 8 with Q = T/8 + 4, so that a warp writing 32
// consecutive coefficients and a warp reading coefficient ci of 32
// consecutive 8-coefficient segments both hit 32 distinct banks.
template <int LR>
struct PColShape
{
	static constexpr int R = 1 << LR, T = PCOL_THREADS, Q = T / 8 + 4, RS = 8 * Q, PS = R * RS;
	static constexpr size_t SMEM = size_t(4) * PS * 4;
	__device__ __forceinline__ static int addr(int k, int c) { return k * RS + (c & 7) * Q + (c >> 3); }
};

// Last LR inverse stages (normalisation folded in), then per 8-coefficient
// segment: CRT of the four primes, base-b digits through the window, and the
// segment's PK_CARRY carries.
template <int LR>
__device__ __forceinline__ void pcol_inv_body(const Args &a, const TestDesc &d, bool dup, uint32_t *sm)
{
	using S = PColShape<LR>;
	constexpr int R = S::R, T = S::T, PS = S::PS, SPR = T / (SEG / 2);
	const size_t Np = size_t(1) << a.n, Cp = size_t(1) << (a.n - LR);
	const size_t c0 = static_cast<size_t>(blockIdx.x) * T;
	const int tid = threadIdx.x;
	for_planes<2>([&](auto PLc) {
		constexpr int PL = decltype(PLc)::value;
		using Z = ZS<2, PL>;
		const uint32_t *src = d.planes + PL * Np + c0 + tid;
		uint32_t x[R];
#pragma unroll
		for (int k = 0; k < R; ++k) x[k] = src[k * Cp];
		inv_reg<Z, LR>(Z{}, x, 1u, a.tab[2].iv[PL], true, __ldg(&a.tab[2].fw[PL][pcol_norm_word(LR)]),
					   __ldg(&a.tab[2].iv[PL][pcol_norm_word(LR)]));
#pragma unroll
		for (int k = 0; k < R; ++k) sm[PL * PS + S::addr(k, tid)] = x[k];
	});
	__syncthreads();
	int32_t *out = d.regs + static_cast<size_t>(a.dst) * (2 * Np);
	for (int e = tid; e < R * SPR; e += T)
	{
		const int k = e / SPR, s = e % SPR;
		const size_t i0 = static_cast<size_t>(k) * Cp + c0 + static_cast<size_t>(s) * (SEG / 2);
		// Garner's digits of the segment's eight coefficients first (independent
		// of one another), then the digit window's dependent chain
		int64_t win[7] = { 0, 0, 0, 0, 0, 0, 0 };
		int32_t dg[SEG];
		uint32_t g[SEG / 2][4];
#pragma unroll
		for (int ci = 0; ci < SEG / 2; ++ci)
		{
#pragma unroll
			for (int pl = 0; pl < 4; ++pl) g[ci][pl] = sm[pl * PS + S::addr(k, s * (SEG / 2) + ci)];
			crt_garner4(g[ci]);
		}
#pragma unroll
		for (int ci = 0; ci < SEG / 2; ++ci)
		{
			crt_window_g(g[ci], dup ? 1 : 0, d.pk, win);
			dg[2 * ci] = window_digit(d.ck, win);
			dg[2 * ci + 1] = window_digit(d.ck, win);
		}
		int4 *o = reinterpret_cast<int4 *>(out + 2 * i0);
#pragma unroll
		for (int i = 0; i < SEG / 4; ++i) o[i] = make_int4(dg[4 * i], dg[4 * i + 1], dg[4 * i + 2], dg[4 * i + 3]);
		int64_t *cs = d.carry + PK_CARRY * (i0 / (SEG / 2));
#pragma unroll
		for (int q = 0; q < PK_CARRY; ++q) cs[q] = win[q];
	}
}

// 16-row columns hold 32 digits and 15 two-word roots per thread: three CTAs
// per SM leave them 85 registers (the inverse kernel's tile fits three anyway).
// 8-row columns at five CTAs per SM (48 registers; 16 bytes spilled in the
// forward kernel): the 64-test n = 16 batch 90.1 -> 89.3 us per squaring
// against four, 93.7 at six (40 registers, 60 bytes spilled).
__host__ __device__ constexpr int pcol_min_blocks(int lr) { return (lr >= 4) ? 3 : 5; }

template <int LR>
__global__ void __launch_bounds__(PCOL_THREADS, pcol_min_blocks(LR)) k_pcol_fwd(const Args a)
{
	pdl_wait();
	__shared__ int32_t sm[(1 << LR) * (2 * PCOL_THREADS + 2 * PCOL_THREADS / SEG)];
	const int t = a.tests[blockIdx.y];
	const TestDesc &d = a.desc[t];
	bool active;
	(void)get_dup(a, d, t, a.j, active);
	if (!active) return;
	pcol_fwd_body<LR>(a, d, sm);
}

template <int LR>
__global__ void __launch_bounds__(PCOL_THREADS, pcol_min_blocks(LR)) k_pcol_inv(const Args a)
{
	pdl_wait();
	extern __shared__ __align__(16) uint32_t sm[];
	const int t = a.tests[blockIdx.y];
	const TestDesc &d = a.desc[t];
	bool active;
	const bool dup = get_dup(a, d, t, a.j, active);
	if (!active) return;
	pcol_inv_body<LR>(a, d, dup, sm);
}

// Plane-split packed columns for batches too small to fill the GPU with one
// thread per packed column: a CTA takes PCS_T columns with a thread per
// (plane, column), 4 PCS_T threads.  The inverse kernel then runs Garner's
// step per coefficient over all threads (digits back into the tile), and the
// digit window per 8-coefficient segment.
constexpr int PCS_T = 64;

template <int LR>
__device__ __forceinline__ void pcol_fwd_split_body(const Args &a, const TestDesc &d, int32_t *sm)
{
	constexpr int R = 1 << LR, T = PCS_T, NT = 4 * T, RW = 2 * T + 2 * T / SEG;
	const size_t Np = size_t(1) << a.n, Cp = size_t(1) << (a.n - LR);
	const size_t c0 = static_cast<size_t>(blockIdx.x) * T;
	const int tid = threadIdx.x, c = tid % T, pl = tid / T;
	int32_t *const srcreg = d.regs + static_cast<size_t>(a.src) * (2 * Np);
	if (a.fix)
	{
		// digit j of row k at k RW + j + j / 16; one thread per 16-digit segment
		for (int e = tid; e < R * T; e += NT)
		{
			const int k = e / T, cc = e % T;
			const int2 v = *reinterpret_cast<const int2 *>(srcreg + 2 * (static_cast<size_t>(k) * Cp + c0 + cc));
			int32_t *p = sm + k * RW + 2 * cc + cc / (SEG / 2);
			p[0] = v.x; p[1] = v.y;
		}
		__syncthreads();
		const size_t nseg = (2 * Np) / SEG;
		for (int e = tid; e < R * (2 * T / SEG); e += NT)
		{
			const int k = e / (2 * T / SEG), s = e % (2 * T / SEG);
			const size_t j0 = 2 * (static_cast<size_t>(k) * Cp + c0) + static_cast<size_t>(s) * SEG;
			fix_segment5(d, sm + k * RW + s * (SEG + 1), srcreg + j0, j0 / SEG, nseg, a.op == OP_FWD, a.err);
		}
		__syncthreads();
	}
	const auto z = prime_rt<2>(pl);
	const uint32_t bb = d.b, bm = d.pk.bm[pl];
	uint32_t x[R];
#pragma unroll
	for (int k = 0; k < R; ++k)
	{
		int32_t v0, v1;
		if (a.fix)
		{
			const int32_t *p = sm + k * RW + 2 * c + c / (SEG / 2);
			v0 = p[0]; v1 = p[1];
		}
		else
		{
			const int2 v = *reinterpret_cast<const int2 *>(srcreg + 2 * (static_cast<size_t>(k) * Cp + c0 + c));
			v0 = v.x; v1 = v.y;
		}
		if constexpr (LR == 3) x[k] = pack_residue(z, pack_value(v0, v1, bb));
		else x[k] = z.add(z.from_int(v0), z.mul(z.from_int(v1), bm));
	}
	fwd_reg<decltype(z), LR>(z, x, 1u, a.tab[2].fw[pl]);
	uint32_t *dst = ((a.op == OP_FWD) ? d.zp : d.planes) + pl * Np + c0 + c;
#pragma unroll
	for (int k = 0; k < R; ++k) dst[k * Cp] = x[k];
}

// Tile of the plane-split inverse: coefficient c of row k at k RS + (c % 8) Q
// + c / 8 with Q = 12, RS = 104: a warp writing 32 consecutive coefficients of
// a row, and a warp reading coefficient ci of the 8 segments of 4 rows, both
// hit 32 distinct banks.
template <int LR>
struct PColShapeS
{
	static constexpr int R = 1 << LR, T = PCS_T, Q = 12, RS = 8 * Q + 8, PS = R * RS;
	static constexpr size_t SMEM = size_t(4) * PS * 4;
	__device__ __forceinline__ static int addr(int k, int c) { return k * RS + (c & 7) * Q + (c >> 3); }
};

template <int LR>
__device__ __forceinline__ void pcol_inv_split_body(const Args &a, const TestDesc &d, bool dup, uint32_t *sm)
{
	using S = PColShapeS<LR>;
	constexpr int R = S::R, T = S::T, NT = 4 * T, PS = S::PS, SPR = T / (SEG / 2);
	const size_t Np = size_t(1) << a.n, Cp = size_t(1) << (a.n - LR);
	const size_t c0 = static_cast<size_t>(blockIdx.x) * T;
	const int tid = threadIdx.x;
	{
		const int c = tid % T, pl = tid / T;
		const auto z = prime_rt<2>(pl);
		const uint32_t *src = d.planes + pl * Np + c0 + c;
		uint32_t x[R];
#pragma unroll
		for (int k = 0; k < R; ++k) x[k] = src[k * Cp];
		inv_reg<decltype(z), LR>(z, x, 1u, a.tab[2].iv[pl], true, __ldg(&a.tab[2].fw[pl][pcol_norm_word(LR)]),
								 __ldg(&a.tab[2].iv[pl][pcol_norm_word(LR)]));
#pragma unroll
		for (int k = 0; k < R; ++k) sm[pl * PS + S::addr(k, c)] = x[k];
	}
	__syncthreads();
	for (int e = tid; e < R * T; e += NT)
	{
		const int k = e / T, c = e % T;
		uint32_t g[4];
#pragma unroll
		for (int pl = 0; pl < 4; ++pl) g[pl] = sm[pl * PS + S::addr(k, c)];
		crt_garner4(g);
#pragma unroll
		for (int pl = 0; pl < 4; ++pl) sm[pl * PS + S::addr(k, c)] = g[pl];
	}
	__syncthreads();
	int32_t *out = d.regs + static_cast<size_t>(a.dst) * (2 * Np);
	for (int e = tid; e < R * SPR; e += NT)
	{
		const int k = e / SPR, s = e % SPR;
		const size_t i0 = static_cast<size_t>(k) * Cp + c0 + static_cast<size_t>(s) * (SEG / 2);
		int64_t win[7] = { 0, 0, 0, 0, 0, 0, 0 };
		int32_t dg[SEG];
#pragma unroll
		for (int ci = 0; ci < SEG / 2; ++ci)
		{
			uint32_t g[4];
#pragma unroll
			for (int pl = 0; pl < 4; ++pl) g[pl] = sm[pl * PS + S::addr(k, s * (SEG / 2) + ci)];
			crt_window_g(g, dup ? 1 : 0, d.pk, win);
			dg[2 * ci] = window_digit(d.ck, win);
			dg[2 * ci + 1] = window_digit(d.ck, win);
		}
		int4 *o = reinterpret_cast<int4 *>(out + 2 * i0);
#pragma unroll
		for (int i = 0; i < SEG / 4; ++i) o[i] = make_int4(dg[4 * i], dg[4 * i + 1], dg[4 * i + 2], dg[4 * i + 3]);
		int64_t *cs = d.carry + PK_CARRY * (i0 / (SEG / 2));
#pragma unroll
		for (int q = 0; q < PK_CARRY; ++q) cs[q] = win[q];
	}
}

// MINB = PCS_MINB_HI caps the registers at 40 for six CTAs per SM, the form
// for large launches; PCS_MINB_LO at 64 for four (with no minimum ptxas
// gave the inverse kernel 80 registers, three CTAs per SM).
constexpr int PCS_MINB_HI = 6, PCS_MINB_LO = 4;

template <int LR, int MINB>
__global__ void __launch_bounds__(4 * PCS_T, MINB) k_pcol_fwd_s(const Args a)
{
	pdl_wait();
	__shared__ int32_t sm[(1 << LR) * (2 * PCS_T + 2 * PCS_T / SEG)];
	const int t = a.tests[blockIdx.y];
	const TestDesc &d = a.desc[t];
	bool active;
	(void)get_dup(a, d, t, a.j, active);
	if (!active) return;
	pcol_fwd_split_body<LR>(a, d, sm);
}

template <int LR, int MINB>
__global__ void __launch_bounds__(4 * PCS_T, MINB) k_pcol_inv_s(const Args a)
{
	pdl_wait();
	__shared__ __align__(16) uint32_t sm[4 * PColShapeS<LR>::PS];
	const int t = a.tests[blockIdx.y];
	const TestDesc &d = a.desc[t];
	bool active;
	const bool dup = get_dup(a, d, t, a.j, active);
	if (!active) return;
	pcol_inv_split_body<LR>(a, d, dup, sm);
}

// Pending packed carries of register a.dst absorbed (a.n = n: digits).
__global__ void __launch_bounds__(256) k_pfixup(const Args a)
{
	pdl_wait();
	const int t = a.tests[blockIdx.y];
	const TestDesc &d = a.desc[t];
	bool active;
	(void)get_dup(a, d, t, a.j, active);
	if (!active) return;
	const size_t N = size_t(1) << a.n;
	const size_t nseg = N / SEG;
	const size_t s = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
	if (s >= nseg) return;
	int64_t c[PK_CARRY];
	take_carry5(d, s, nseg, c);
	bool any = false;
#pragma unroll
	for (int k = 0; k < PK_CARRY; ++k) any |= (c[k] != 0);
	if (!any) return;
	int4 *p = reinterpret_cast<int4 *>(d.regs + static_cast<size_t>(a.dst) * N + s * SEG);
	int32_t dg[SEG];
#pragma unroll
	for (int i = 0; i < SEG / 4; ++i)
	{
		const int4 v = p[i];
		dg[4 * i] = v.x; dg[4 * i + 1] = v.y; dg[4 * i + 2] = v.z; dg[4 * i + 3] = v.w;
	}
	if (!absorb5<SEG>(dg, c, d.ck)) atomicOr(a.err, 1u);
#pragma unroll
	for (int i = 0; i < SEG / 4; ++i) p[i] = make_int4(dg[4 * i], dg[4 * i + 1], dg[4 * i + 2], dg[4 * i + 3]);
}

// Each segment absorbs the carry of the previous one (segment 0 takes minus
// the last carry: b^N = -1).
__global__ void __launch_bounds__(256) k_fixup(const Args a)
{
	pdl_wait();
	const int t = a.tests[blockIdx.y];
	const TestDesc &d = a.desc[t];
	bool active;
	(void)get_dup(a, d, t, a.j, active);
	if (!active) return;
	const size_t N = size_t(1) << a.n;
	const size_t nseg = N / SEG;
	const size_t s = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
	if (s >= nseg) return;
	const int64_t cin = take_carry(d, s, nseg);
	if (cin == 0) return;
	int4 *p = reinterpret_cast<int4 *>(d.regs + static_cast<size_t>(a.dst) * N + s * SEG);
	int32_t dg[SEG];
#pragma unroll
	for (int i = 0; i < SEG / 4; ++i)
	{
		const int4 v = p[i];
		dg[4 * i] = v.x; dg[4 * i + 1] = v.y; dg[4 * i + 2] = v.z; dg[4 * i + 3] = v.w;
	}
	if (!absorb<SEG>(dg, cin, d.ck)) atomicOr(a.err, 1u);
#pragma unroll
	for (int i = 0; i < SEG / 4; ++i) p[i] = make_int4(dg[4 * i], dg[4 * i + 1], dg[4 * i + 2], dg[4 * i + 3]);
}

// r_dst = m r_dst digit by digit, carrying inside 16-digit segments and leaving
// the segment carries for k_fixup: the digit-times-scalar step of
// transform::squareMul (src/transformCPUi32.h:774-797).  |digit m| < 2^62.
__global__ void __launch_bounds__(256) k_mulscalar(const Args a, int32_t m)
{
	pdl_wait();
	const int t = a.tests[blockIdx.y];
	if (!test_ok(a, t)) return;
	const TestDesc &d = a.desc[t];
	const size_t N = size_t(1) << a.n;
	const size_t s = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
	if (s >= N / SEG) return;
	int4 *p = reinterpret_cast<int4 *>(d.regs + static_cast<size_t>(a.dst) * N + s * SEG);
	int32_t dg[SEG];
#pragma unroll
	for (int i = 0; i < SEG / 4; ++i)
	{
		const int4 v = p[i];
		dg[4 * i] = v.x; dg[4 * i + 1] = v.y; dg[4 * i + 2] = v.z; dg[4 * i + 3] = v.w;
	}
	int64_t c = 0;
#pragma unroll
	for (int i = 0; i < SEG; ++i) dg[i] = carry_wide(static_cast<int64_t>(dg[i]) * m + c, d.ck, c);
#pragma unroll
	for (int i = 0; i < SEG / 4; ++i) p[i] = make_int4(dg[4 * i], dg[4 * i + 1], dg[4 * i + 2], dg[4 * i + 3]);
	d.carry[s] = c;
}

// ------------------------------------------------------------------ utilities

// reg[dst] = a (digit 0), 0 elsewhere, for every test of the launch.
__global__ void k_set(const Args a, int32_t value)
{
	pdl_wait();
	const int t = a.tests[blockIdx.y];
	if (!test_ok(a, t)) return;
	const size_t N = size_t(1) << a.n;
	int32_t *r = a.desc[t].regs + static_cast<size_t>(a.dst) * N;
	for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < N; i += size_t(gridDim.x) * blockDim.x)
		r[i] = (i == 0) ? value : 0;
}

// Digits loaded into a test's planes (its transform scratch, N words at
// d.planes) checked against |d| <= b/2 + 1: any digit outside sets *bad.
// blockIdx.y = test, four digits per thread.
__global__ void __launch_bounds__(256) k_check_digits(const TestDesc *desc, int n, uint32_t *bad)
{
	const TestDesc &d = desc[blockIdx.y];
	const size_t N = size_t(1) << n;
	const uint32_t lim = d.b / 2 + 1, span = 2 * lim;
	const int4 *src = reinterpret_cast<const int4 *>(d.planes);
	uint32_t out = 0;
	for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < N / 4; i += size_t(gridDim.x) * blockDim.x)
	{
		const int4 v = src[i];
		out |= static_cast<uint32_t>(static_cast<uint32_t>(v.x) + lim > span) |
			   static_cast<uint32_t>(static_cast<uint32_t>(v.y) + lim > span) |
			   static_cast<uint32_t>(static_cast<uint32_t>(v.z) + lim > span) |
			   static_cast<uint32_t>(static_cast<uint32_t>(v.w) + lim > span);
	}
	if (__any_sync(0xffffffffu, out != 0) && ((threadIdx.x & 31) == 0)) atomicOr(bad, 1u);
}

// Register reg of every test <- the digits staged in its planes, unless *bad
// (then every register stays as it was).
__global__ void __launch_bounds__(256) k_commit_digits(const TestDesc *desc, int n, int reg, const uint32_t *bad)
{
	if (*bad != 0) return;
	const TestDesc &d = desc[blockIdx.y];
	const size_t N = size_t(1) << n;
	const int4 *src = reinterpret_cast<const int4 *>(d.planes);
	int4 *dst = reinterpret_cast<int4 *>(d.regs + static_cast<size_t>(reg) * N);
	for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < N / 4; i += size_t(gridDim.x) * blockDim.x)
		dst[i] = src[i];
}

// reg[dst] = reg[src] for every test of the launch.
__global__ void k_copy(const Args a)
{
	pdl_wait();
	const int t = a.tests[blockIdx.y];
	if (!test_ok(a, t)) return;
	const size_t N = size_t(1) << a.n;
	const int4 *s = reinterpret_cast<const int4 *>(a.desc[t].regs + static_cast<size_t>(a.src) * N);
	int4 *o = reinterpret_cast<int4 *>(a.desc[t].regs + static_cast<size_t>(a.dst) * N);
	for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < N / 4; i += size_t(gridDim.x) * blockDim.x)
		o[i] = s[i];
}

// Root tables of one prime p for length N = 2^n, in the layout load_twiddles
// reads (gf_ntt.cuh): entry k >= 1 of fw is psi^e and of iv is psi^-e, with
// e = bitrev_n(k) and psi a primitive 2N-th root of unity; one word per entry
// in Montgomery form (words = 1, the 32-bit primes) or the root in normal form
// followed by its Shoup quotient floor(w 2^32 / p) (words = 2).  A thread
// walks `run` consecutive exponents e, one product by psi (and by psi^-1) per
// entry, and writes entry bitrev_n(e).  Entry 0 holds the normalisation
// constants c (fw) and k0 (iv) computed by the host.  Exact integer
// arithmetic: the same words as a host-side build.
__device__ __forceinline__ uint32_t mulmod_u64(uint32_t a, uint32_t b, uint32_t p)
{
	return static_cast<uint32_t>((static_cast<uint64_t>(a) * b) % p);
}

__device__ __forceinline__ void put_root_d(uint32_t *t, uint32_t k, uint32_t w, uint32_t p, int words)
{
	if (words == 1) t[k] = static_cast<uint32_t>((static_cast<uint64_t>(w) << 32) % p);
	else
	{
		t[2 * k] = w;
		t[2 * k + 1] = static_cast<uint32_t>((static_cast<uint64_t>(w) << 32) / p);
	}
}

__global__ void k_roots(uint32_t *fw, uint32_t *iv, uint32_t p, uint32_t psi, uint32_t psi_inv, int n, int words, int run,
						uint32_t c, uint32_t k0, uint32_t c2, uint32_t k02)
{
	const uint32_t N = 1u << n;
	const uint32_t e0 = (blockIdx.x * blockDim.x + threadIdx.x) * static_cast<uint32_t>(run);
	if (e0 >= N) return;
	// psi^e0 and psi^-e0 by square-and-multiply
	uint32_t w = 1, wi = 1, y = psi, yi = psi_inv;
	for (uint32_t e = e0; e != 0; e >>= 1)
	{
		if (e & 1) { w = mulmod_u64(w, y, p); wi = mulmod_u64(wi, yi, p); }
		y = mulmod_u64(y, y, p);
		yi = mulmod_u64(yi, yi, p);
	}
	for (uint32_t e = e0; (e < e0 + static_cast<uint32_t>(run)) && (e < N); ++e)
	{
		if (e == 0)
		{
			fw[0] = c;
			iv[0] = k0;
			if (words == 2) { fw[1] = c2; iv[1] = k02; }
		}
		else
		{
			const uint32_t k = __brev(e) >> (32 - n);
			put_root_d(fw, k, w, p, words);
			put_root_d(iv, k, wi, p, words);
		}
		w = mulmod_u64(w, psi, p);
		wi = mulmod_u64(wi, psi_inv, p);
	}
}

__device__ __forceinline__ uint32_t powmod_d(uint32_t a, uint64_t e, uint32_t p)
{
	uint32_t r = 1;
	for (; e != 0; e >>= 1)
	{
		if (e & 1) r = mulmod_u64(r, a, p);
		a = mulmod_u64(a, a, p);
	}
	return r;
}

// Twist tables of one prime for a six-step split of 2^n points into R = 2^lr
// rows (twist_regs): thread i < 16 C writes H[m][c] (i = m C + c) of both
// directions, threads m = 0 also G[c].  words: root entry size.
__global__ void k_twist(uint32_t *tf, uint32_t *ti, uint32_t p, uint32_t psi, uint32_t psi_inv, int n, int lr, int words)
{
	const uint32_t C = 1u << (n - lr);
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= 16 * C) return;
	const uint32_t m = i / C, c = i % C;
	const uint64_t two_n = uint64_t(2) << n;
	const uint64_t bm = __brev(m) >> 28;
	const uint64_t e = (uint64_t(c) * (2 * bm + 1) + two_n - ((uint64_t(c) << lr) % two_n)) % two_n;
	const uint32_t r1 = static_cast<uint32_t>((uint64_t(1) << 32) % p);
	tf[i] = mulmod_u64(powmod_d(psi, e, p), r1, p);
	ti[i] = mulmod_u64(powmod_d(psi_inv, e, p), r1, p);
	if (m == 0)
	{
		const uint64_t g = (32ull * c) % two_n;
		put_root_d(tf + 16 * C, c, powmod_d(psi, g, p), p, words);
		put_root_d(ti + 16 * C, c, powmod_d(psi_inv, g, p), p, words);
	}
}

// pos[t] = max(pos[t] - count, -1) for every test (end of a four-step block;
// k_small advances its own tests the same way).
__global__ void k_pos_sub(int64_t *pos, const int32_t *tests, int ntests, int count)
{
	pdl_wait();
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if ((i < ntests) && (static_cast<uint32_t>(tests[i]) < static_cast<uint32_t>(ntests)))
	{
		const int64_t p = pos[tests[i]] - count;
		pos[tests[i]] = (p < -1) ? -1 : p;
	}
}

}  // namespace gfc
