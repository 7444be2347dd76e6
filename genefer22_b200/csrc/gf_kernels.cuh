// gf_kernels.cuh -- sm_100a kernels of the modular-squaring engine.
//
// One squaring r <- r^2 (or 2 r^2) mod (b^N + 1), N = 2^n, is: digits ->
// residues in W prime planes -> forward negacyclic NTT -> pointwise square
// -> inverse NTT (normalisation folded into the last stage) -> CRT ->
// base-b carry.  This is the work of genefer's transform::squareDup
// (src/transform.h:59; CPU reference src/transformCPUi32.h:857-868).
//
// Resting state of a register: N signed int32 digits in natural order with
// |d| <= b/2 + 1 (balanced).  Two kernel shapes:
//   * k_small (n <= 14): one CTA owns one test; the W planes live in shared
//     memory and the CTA can run many squarings without touching HBM.
//   * four-step (n >= 15): N = R x C.  k_col_fwd does the first log2 R stages
//     on column tiles, k_row the remaining stages + pointwise + inverse on
//     rows, k_col_inv the last inverse stages, CRT and the carry inside
//     16-digit segments, and k_fixup adds each segment's carry to the next.
#pragma once

#include <type_traits>
#include "gf_ntt.cuh"

namespace gfc {

enum : int { OP_SQUARE = 0, OP_MUL = 1, OP_FWD = 2 };
enum : int { DUP_NONE = 0, DUP_ALL = 1, DUP_BITS = 2 };

constexpr int SEG = 16;          // digits per carry segment
constexpr int SMALL_MAX_LOGN = 14;

struct TestDesc
{
	int32_t *regs;          // num_regs x N digits
	uint32_t *planes;       // 3 x N transform scratch
	uint32_t *zp;           // 3 x N multiplicand (transform domain, normal form)
	int64_t *carry;         // N / SEG segment carries
	const uint32_t *ebits;  // exponent bits, bit i in word i/32 (may be null)
	uint64_t binv;          // floor((2^64 - 1) / b)
	uint32_t b;
	int32_t set;            // prime set: 0 (W = 2), 1 (W = 3)
};

struct Tables
{
	const uint32_t *fw[3];  // forward roots, Montgomery form; fw[p][0] = normalisation c
	const uint32_t *iv[3];  // inverse roots, Montgomery form; iv[p][0] = K (last stage)
};

struct Args
{
	const TestDesc *desc;   // all tests of the batch
	const int32_t *tests;   // indices of the tests this launch serves
	int64_t *pos;           // per-test current exponent bit index
	uint32_t *err;          // error flags (bit 0: carry not absorbed)
	Tables tab;
	int n, lr;              // log2 N, log2 R (four-step)
	int num_regs, src, dst; // registers
	int op, dup_mode, count, j;  // operation, dup source, squarings (k_small), squaring index in block
};

template <int SET, int PL>
using ZS = Zp<PrimeSet<SET>::p[PL], PrimeSet<SET>::P31>;

template <int SET, class F>
__device__ __forceinline__ void for_planes(F &&f)
{
	f(std::integral_constant<int, 0>{});
	f(std::integral_constant<int, 1>{});
	if constexpr (PrimeSet<SET>::W == 3) f(std::integral_constant<int, 2>{});
}

__device__ __forceinline__ bool exp_bit(const uint32_t *ebits, int64_t i)
{
	return ((__ldg(&ebits[i >> 5]) >> (i & 31)) & 1u) != 0;
}

// dup flag of squaring j (DUP_BITS: bit pos - j of the exponent); false with
// `active` cleared when the test has no squaring left.
__device__ __forceinline__ bool get_dup(const Args &a, const TestDesc &d, int t, int j, bool &active)
{
	active = true;
	if (a.dup_mode == DUP_BITS)
	{
		const int64_t i = a.pos[t] - j;
		if (i < 0) { active = false; return false; }
		return exp_bit(d.ebits, i);
	}
	return a.dup_mode == DUP_ALL;
}

// Adds carry `c` to the digits of one segment: reduces while |c| > 1, then
// leaves the last +-1 in the next digit unreduced (|digit| <= b/2 + 1).
template <int D>
__device__ __forceinline__ bool absorb(int32_t (&dg)[D], int64_t c, uint32_t b, uint64_t binv)
{
	bool active = (c != 0);
#pragma unroll
	for (int k = 0; k < D; ++k)
	{
		if (active)
		{
			if ((c > 1) || (c < -1))
			{
				int64_t q;
				dg[k] = digit_carry64(static_cast<int64_t>(dg[k]) + c, b, binv, q);
				c = q;
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

// ------------------------------------------------------------------ passes

template <int SET, int PL, int r, class Map>
__device__ __forceinline__ void pass_fwd(uint32_t *buf, const Map &mp, int l, int sigma, int lanes_log, bool lane_fast,
										 uint32_t base0, uint32_t base_step, const uint32_t *__restrict__ tw)
{
	using Z = ZS<SET, PL>;
	const int groups_log = l - r;
	const int items = 1 << (lanes_log + groups_log);
	for (int it = threadIdx.x; it < items; it += blockDim.x)
	{
		int lane, g;
		if (lane_fast) { lane = it & ((1 << lanes_log) - 1); g = it >> lanes_log; }
		else { g = it & ((1 << groups_log) - 1); lane = it >> groups_log; }
		const Group G(g, l, sigma, r);
		uint32_t x[1 << r];
#pragma unroll
		for (int m = 0; m < (1 << r); ++m) x[m] = buf[mp(G.i0 + m * G.step, lane)];
		const uint32_t base = base0 + static_cast<uint32_t>(lane) * base_step;
		fwd_reg<Z, r>(x, (base << sigma) + G.blk, tw);
#pragma unroll
		for (int m = 0; m < (1 << r); ++m) buf[mp(G.i0 + m * G.step, lane)] = x[m];
	}
}

template <int SET, int PL, int r, class Map>
__device__ __forceinline__ void pass_inv(uint32_t *buf, const Map &mp, int l, int sigma, int lanes_log, bool lane_fast,
										 uint32_t base0, uint32_t base_step, const uint32_t *__restrict__ tw,
										 const uint32_t *__restrict__ twi)
{
	using Z = ZS<SET, PL>;
	const int groups_log = l - r;
	const int items = 1 << (lanes_log + groups_log);
	const uint32_t c_norm = __ldg(&tw[0]), k_norm = __ldg(&twi[0]);
	for (int it = threadIdx.x; it < items; it += blockDim.x)
	{
		int lane, g;
		if (lane_fast) { lane = it & ((1 << lanes_log) - 1); g = it >> lanes_log; }
		else { g = it & ((1 << groups_log) - 1); lane = it >> groups_log; }
		const Group G(g, l, sigma, r);
		uint32_t x[1 << r];
#pragma unroll
		for (int m = 0; m < (1 << r); ++m) x[m] = buf[mp(G.i0 + m * G.step, lane)];
		const uint32_t base = base0 + static_cast<uint32_t>(lane) * base_step;
		const uint32_t tb = (base << sigma) + G.blk;
		inv_reg<Z, r>(x, tb, twi, tb == 1u, c_norm, k_norm);
#pragma unroll
		for (int m = 0; m < (1 << r); ++m) buf[mp(G.i0 + m * G.step, lane)] = x[m];
	}
}

// Last forward pass + pointwise square (or product with the multiplicand) +
// first inverse pass, without leaving registers.  `zrow` points at the
// multiplicand plane at this tile's first element (row layout only).
template <int SET, int PL, int r, class Map>
__device__ __forceinline__ void pass_mid(uint32_t *buf, const Map &mp, int l, int sigma, int lanes_log,
										 uint32_t base0, uint32_t base_step, const uint32_t *__restrict__ tw,
										 const uint32_t *__restrict__ twi, const uint32_t *__restrict__ zrow, bool is_mul)
{
	using Z = ZS<SET, PL>;
	const int groups_log = l - r;
	const int items = 1 << (lanes_log + groups_log);
	const uint32_t c_norm = __ldg(&tw[0]), k_norm = __ldg(&twi[0]);
	for (int it = threadIdx.x; it < items; it += blockDim.x)
	{
		const int g = it & ((1 << groups_log) - 1), lane = it >> groups_log;
		const Group G(g, l, sigma, r);
		uint32_t x[1 << r];
#pragma unroll
		for (int m = 0; m < (1 << r); ++m) x[m] = buf[mp(G.i0 + m * G.step, lane)];
		const uint32_t base = base0 + static_cast<uint32_t>(lane) * base_step;
		const uint32_t tb = (base << sigma) + G.blk;
		fwd_reg<Z, r>(x, tb, tw);
		if (is_mul)
		{
#pragma unroll
			for (int m = 0; m < (1 << r); ++m) x[m] = Z::mul(x[m], __ldg(&zrow[(lane << l) + G.i0 + m * G.step]));
		}
		else
		{
#pragma unroll
			for (int m = 0; m < (1 << r); ++m) x[m] = Z::mul(x[m], x[m]);
		}
		inv_reg<Z, r>(x, tb, twi, tb == 1u, c_norm, k_norm);
#pragma unroll
		for (int m = 0; m < (1 << r); ++m) buf[mp(G.i0 + m * G.step, lane)] = x[m];
	}
}

// Radix schedule: passes of 4 stages, the last one takes the remainder.
__host__ __device__ constexpr int num_passes(int l) { return (l + 3) / 4; }
__host__ __device__ constexpr int pass_r(int l, int p) { return (p < l / 4) ? 4 : (l % 4); }

template <int SET, int PL, class Map>
__device__ __forceinline__ void run_fwd(uint32_t *buf, const Map &mp, int l, int lanes_log, bool lane_fast, uint32_t base0,
										uint32_t base_step, const uint32_t *tw, int npass)
{
	int sigma = 0;
	for (int p = 0; p < npass; ++p)
	{
		const int r = pass_r(l, p);
		switch (r)
		{
			case 4: pass_fwd<SET, PL, 4>(buf, mp, l, sigma, lanes_log, lane_fast, base0, base_step, tw); break;
			case 3: pass_fwd<SET, PL, 3>(buf, mp, l, sigma, lanes_log, lane_fast, base0, base_step, tw); break;
			case 2: pass_fwd<SET, PL, 2>(buf, mp, l, sigma, lanes_log, lane_fast, base0, base_step, tw); break;
			default: pass_fwd<SET, PL, 1>(buf, mp, l, sigma, lanes_log, lane_fast, base0, base_step, tw); break;
		}
		sigma += r;
		__syncthreads();
	}
}

// Inverse passes p = npass-1 .. 0 (stages in reverse order).
template <int SET, int PL, class Map>
__device__ __forceinline__ void run_inv(uint32_t *buf, const Map &mp, int l, int lanes_log, bool lane_fast, uint32_t base0,
										uint32_t base_step, const uint32_t *tw, const uint32_t *twi, int npass)
{
	int sigma = 0;
	for (int p = 0; p < npass; ++p) sigma += pass_r(l, p);
	for (int p = npass - 1; p >= 0; --p)
	{
		const int r = pass_r(l, p);
		sigma -= r;
		switch (r)
		{
			case 4: pass_inv<SET, PL, 4>(buf, mp, l, sigma, lanes_log, lane_fast, base0, base_step, tw, twi); break;
			case 3: pass_inv<SET, PL, 3>(buf, mp, l, sigma, lanes_log, lane_fast, base0, base_step, tw, twi); break;
			case 2: pass_inv<SET, PL, 2>(buf, mp, l, sigma, lanes_log, lane_fast, base0, base_step, tw, twi); break;
			default: pass_inv<SET, PL, 1>(buf, mp, l, sigma, lanes_log, lane_fast, base0, base_step, tw, twi); break;
		}
		__syncthreads();
	}
}

// Full squaring/product core on `lanes` row transforms of length 2^l held in
// shared memory: forward, pointwise, inverse.
template <int SET, int PL>
__device__ __forceinline__ void row_core(uint32_t *buf, const RowMap &mp, int l, int lanes_log, uint32_t base0,
										 const uint32_t *tw, const uint32_t *twi, const uint32_t *zrow, int op)
{
	const int np = num_passes(l);
	if (op == OP_FWD) { run_fwd<SET, PL>(buf, mp, l, lanes_log, false, base0, 1u, tw, np); return; }
	run_fwd<SET, PL>(buf, mp, l, lanes_log, false, base0, 1u, tw, np - 1);
	int sigma = 0;
	for (int p = 0; p < np - 1; ++p) sigma += pass_r(l, p);
	const int r = pass_r(l, np - 1);
	const bool is_mul = (op == OP_MUL);
	switch (r)
	{
		case 4: pass_mid<SET, PL, 4>(buf, mp, l, sigma, lanes_log, base0, 1u, tw, twi, zrow, is_mul); break;
		case 3: pass_mid<SET, PL, 3>(buf, mp, l, sigma, lanes_log, base0, 1u, tw, twi, zrow, is_mul); break;
		case 2: pass_mid<SET, PL, 2>(buf, mp, l, sigma, lanes_log, base0, 1u, tw, twi, zrow, is_mul); break;
		default: pass_mid<SET, PL, 1>(buf, mp, l, sigma, lanes_log, base0, 1u, tw, twi, zrow, is_mul); break;
	}
	__syncthreads();
	// remaining inverse passes np-2 .. 0
	for (int p = np - 2; p >= 0; --p)
	{
		const int rr = pass_r(l, p);
		sigma -= rr;
		switch (rr)
		{
			case 4: pass_inv<SET, PL, 4>(buf, mp, l, sigma, lanes_log, false, base0, 1u, tw, twi); break;
			case 3: pass_inv<SET, PL, 3>(buf, mp, l, sigma, lanes_log, false, base0, 1u, tw, twi); break;
			case 2: pass_inv<SET, PL, 2>(buf, mp, l, sigma, lanes_log, false, base0, 1u, tw, twi); break;
			default: pass_inv<SET, PL, 1>(buf, mp, l, sigma, lanes_log, false, base0, 1u, tw, twi); break;
		}
		__syncthreads();
	}
}

// ------------------------------------------------------------------ k_small

// Shared memory: W planes of N (+N/32 padding) words, then T int64 carries.
template <int SET, int LOGN, int T>
__global__ void __launch_bounds__(T, 1) k_small(const Args a)
{
	constexpr int W = PrimeSet<SET>::W;
	constexpr int N = 1 << LOGN;
	constexpr int D = N / T;           // digits per thread (multiple of SEG)
	constexpr int PN = N + N / 32;
	static_assert(D % SEG == 0, "digits per thread");
	extern __shared__ __align__(16) uint32_t sm[];
	int64_t *const sc = reinterpret_cast<int64_t *>(sm + W * PN);

	const int t = a.tests[blockIdx.x];
	const TestDesc &d = a.desc[t];
	const int tid = threadIdx.x;
	const uint32_t b = d.b;
	const uint64_t binv = d.binv;
	const RowMap mp{LOGN};

	int32_t dg[D];
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
		bool active;
		const bool dup = (a.op == OP_SQUARE) ? get_dup(a, d, t, it, active) : (active = true, false);
		if (!active) break;

		for_planes<SET>([&](auto PLc) {
			constexpr int PL = decltype(PLc)::value;
			using Z = ZS<SET, PL>;
			uint32_t *pl = sm + PL * PN;
#pragma unroll
			for (int i = 0; i < D; ++i) pl[mp(tid * D + i, 0)] = Z::from_int(dg[i]);
		});
		__syncthreads();

		for_planes<SET>([&](auto PLc) {
			constexpr int PL = decltype(PLc)::value;
			row_core<SET, PL>(sm + PL * PN, mp, LOGN, 0, 1u, a.tab.fw[PL], a.tab.iv[PL], d.zp + PL * N, a.op);
		});

		if (a.op == OP_FWD)
		{
			for_planes<SET>([&](auto PLc) {
				constexpr int PL = decltype(PLc)::value;
				const uint32_t *pl = sm + PL * PN;
				uint32_t *zo = d.zp + PL * N;
				for (int i = tid; i < N; i += T) zo[i] = pl[mp(i, 0)];
			});
			return;
		}

		// CRT + carry over this thread's D consecutive digits.
		int64_t c = 0;
#pragma unroll
		for (int i = 0; i < D; ++i)
		{
			uint32_t x[3];
			for_planes<SET>([&](auto PLc) {
				constexpr int PL = decltype(PLc)::value;
				x[PL] = sm[PL * PN + mp(tid * D + i, 0)];
			});
			i128 v = crt<SET>(x);
			if (dup) v += v;
			dg[i] = digit_carry(v + c, b, binv, c);
		}
		sc[tid] = c;
		__syncthreads();
		const int64_t cin = (tid == 0) ? -sc[T - 1] : sc[tid - 1];
		if (!absorb<D>(dg, cin, b, binv)) atomicOr(a.err, 1u);
		__syncthreads();
		++done;
	}

	{
		int4 *dst = reinterpret_cast<int4 *>(d.regs + static_cast<size_t>(a.dst) * N + tid * D);
#pragma unroll
		for (int i = 0; i < D / 4; ++i) dst[i] = make_int4(dg[4 * i], dg[4 * i + 1], dg[4 * i + 2], dg[4 * i + 3]);
	}
	if ((tid == 0) && (a.op == OP_SQUARE) && (a.dup_mode == DUP_BITS)) a.pos[t] -= done;
}

// ------------------------------------------------------------------ four-step

__host__ __device__ constexpr int col_width(int lr) { return (lr >= 10) ? 16 : ((4096 >> lr) > 32 ? (4096 >> lr) : 32); }
__host__ __device__ constexpr int col_stride(int lr) { return (col_width(lr) == 16) ? 17 : col_width(lr); }

// Columns: tile of cw columns x R rows; first log2 R forward stages.
template <int SET, int LR>
__global__ void __launch_bounds__(256) k_col_fwd(const Args a)
{
	constexpr int R = 1 << LR, CW = col_width(LR), RS = col_stride(LR);
	constexpr int CWL = (CW == 16) ? 4 : ((CW == 32) ? 5 : ((CW == 64) ? 6 : ((CW == 128) ? 7 : ((CW == 256) ? 8 : 9))));
	extern __shared__ __align__(16) uint32_t sm[];
	const int t = a.tests[blockIdx.y];
	const TestDesc &d = a.desc[t];
	bool active;
	(void)get_dup(a, d, t, a.j, active);
	if (!active) return;
	const int n = a.n, lc = n - LR;
	const size_t N = size_t(1) << n, C = size_t(1) << lc;
	const int c0 = blockIdx.x * CW;
	const int32_t *src = d.regs + static_cast<size_t>(a.src) * N;
	uint32_t *dst = (a.op == OP_FWD) ? d.zp : d.planes;

	for (int e = threadIdx.x; e < R * CW; e += blockDim.x)
	{
		const int k = e >> CWL, cc = e & (CW - 1);
		const int32_t dv = src[static_cast<size_t>(k) * C + c0 + cc];
		for_planes<SET>([&](auto PLc) {
			constexpr int PL = decltype(PLc)::value;
			sm[PL * R * RS + k * RS + cc] = ZS<SET, PL>::from_int(dv);
		});
	}
	__syncthreads();
	const ColMap mp{RS};
	for_planes<SET>([&](auto PLc) {
		constexpr int PL = decltype(PLc)::value;
		run_fwd<SET, PL>(sm + PL * R * RS, mp, LR, CWL, true, 1u, 0u, a.tab.fw[PL], num_passes(LR));
	});
	for (int e = threadIdx.x; e < R * CW; e += blockDim.x)
	{
		const int k = e >> CWL, cc = e & (CW - 1);
		for_planes<SET>([&](auto PLc) {
			constexpr int PL = decltype(PLc)::value;
			dst[PL * N + static_cast<size_t>(k) * C + c0 + cc] = sm[PL * R * RS + k * RS + cc];
		});
	}
}

// Rows: the last log2 C forward stages, pointwise, first inverse stages.
template <int SET, int LC>
__global__ void __launch_bounds__(256) k_row(const Args a)
{
	constexpr int C = 1 << LC;
	constexpr int PC = C + C / 32;
	extern __shared__ __align__(16) uint32_t sm[];
	const int t = a.tests[blockIdx.y];
	const TestDesc &d = a.desc[t];
	bool active;
	(void)get_dup(a, d, t, a.j, active);
	if (!active) return;
	const int n = a.n, lr = n - LC;
	const size_t N = size_t(1) << n;
	const int k = blockIdx.x;             // one row per CTA
	uint32_t *buf = (a.op == OP_FWD) ? d.zp : d.planes;
	const RowMap mp{LC};

	for_planes<SET>([&](auto PLc) {
		constexpr int PL = decltype(PLc)::value;
		const uint32_t *row = buf + PL * N + static_cast<size_t>(k) * C;
		for (int i = threadIdx.x; i < C; i += blockDim.x) sm[PL * PC + mp(i, 0)] = row[i];
	});
	__syncthreads();
	for_planes<SET>([&](auto PLc) {
		constexpr int PL = decltype(PLc)::value;
		row_core<SET, PL>(sm + PL * PC, mp, LC, 0, (1u << lr) + static_cast<uint32_t>(k), a.tab.fw[PL], a.tab.iv[PL],
						  d.zp + PL * N + static_cast<size_t>(k) * C, a.op);
	});
	for_planes<SET>([&](auto PLc) {
		constexpr int PL = decltype(PLc)::value;
		uint32_t *row = buf + PL * N + static_cast<size_t>(k) * C;
		for (int i = threadIdx.x; i < C; i += blockDim.x) row[i] = sm[PL * PC + mp(i, 0)];
	});
}

// Columns: last log2 R inverse stages, CRT, carry inside 16-digit segments.
template <int SET, int LR>
__global__ void __launch_bounds__(256) k_col_inv(const Args a)
{
	constexpr int R = 1 << LR, CW = col_width(LR), RS = col_stride(LR);
	constexpr int CWL = (CW == 16) ? 4 : ((CW == 32) ? 5 : ((CW == 64) ? 6 : ((CW == 128) ? 7 : ((CW == 256) ? 8 : 9))));
	constexpr int SPR = CW / SEG;        // segments per tile row
	extern __shared__ __align__(16) uint32_t sm[];
	const int t = a.tests[blockIdx.y];
	const TestDesc &d = a.desc[t];
	bool active;
	const bool dup = get_dup(a, d, t, a.j, active);
	if (!active) return;
	const int n = a.n, lc = n - LR;
	const size_t N = size_t(1) << n, C = size_t(1) << lc;
	const int c0 = blockIdx.x * CW;
	const uint32_t b = d.b;
	const uint64_t binv = d.binv;

	for (int e = threadIdx.x; e < R * CW; e += blockDim.x)
	{
		const int k = e >> CWL, cc = e & (CW - 1);
		for_planes<SET>([&](auto PLc) {
			constexpr int PL = decltype(PLc)::value;
			sm[PL * R * RS + k * RS + cc] = d.planes[PL * N + static_cast<size_t>(k) * C + c0 + cc];
		});
	}
	__syncthreads();
	const ColMap mp{RS};
	for_planes<SET>([&](auto PLc) {
		constexpr int PL = decltype(PLc)::value;
		run_inv<SET, PL>(sm + PL * R * RS, mp, LR, CWL, true, 1u, 0u, a.tab.fw[PL], a.tab.iv[PL], num_passes(LR));
	});

	int32_t *out = d.regs + static_cast<size_t>(a.dst) * N;
	for (int e = threadIdx.x; e < R * SPR; e += blockDim.x)
	{
		const int k = e / SPR, s = e % SPR;
		const size_t j0 = static_cast<size_t>(k) * C + c0 + s * SEG;
		int64_t c = 0;
		int32_t dg[SEG];
#pragma unroll
		for (int i = 0; i < SEG; ++i)
		{
			uint32_t x[3];
			for_planes<SET>([&](auto PLc) {
				constexpr int PL = decltype(PLc)::value;
				x[PL] = sm[PL * R * RS + k * RS + s * SEG + i];
			});
			i128 v = crt<SET>(x);
			if (dup) v += v;
			dg[i] = digit_carry(v + c, b, binv, c);
		}
		int4 *o = reinterpret_cast<int4 *>(out + j0);
#pragma unroll
		for (int i = 0; i < SEG / 4; ++i) o[i] = make_int4(dg[4 * i], dg[4 * i + 1], dg[4 * i + 2], dg[4 * i + 3]);
		d.carry[j0 / SEG] = c;
	}
}

// Each segment absorbs the carry of the previous one (segment 0 takes minus
// the last carry: b^N = -1).
__global__ void __launch_bounds__(256) k_fixup(const Args a)
{
	const int t = a.tests[blockIdx.y];
	const TestDesc &d = a.desc[t];
	bool active;
	(void)get_dup(a, d, t, a.j, active);
	if (!active) return;
	const size_t N = size_t(1) << a.n;
	const size_t nseg = N / SEG;
	const size_t s = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
	if (s >= nseg) return;
	const int64_t cin = (s == 0) ? -d.carry[nseg - 1] : d.carry[s - 1];
	if (cin == 0) return;
	int4 *p = reinterpret_cast<int4 *>(d.regs + static_cast<size_t>(a.dst) * N + s * SEG);
	int32_t dg[SEG];
#pragma unroll
	for (int i = 0; i < SEG / 4; ++i)
	{
		const int4 v = p[i];
		dg[4 * i] = v.x; dg[4 * i + 1] = v.y; dg[4 * i + 2] = v.z; dg[4 * i + 3] = v.w;
	}
	if (!absorb<SEG>(dg, cin, d.b, d.binv)) atomicOr(a.err, 1u);
#pragma unroll
	for (int i = 0; i < SEG / 4; ++i) p[i] = make_int4(dg[4 * i], dg[4 * i + 1], dg[4 * i + 2], dg[4 * i + 3]);
}

// ------------------------------------------------------------------ utilities

// reg[dst] = a (digit 0), 0 elsewhere, for every test of the launch.
__global__ void k_set(const Args a, int32_t value)
{
	const int t = a.tests[blockIdx.y];
	const size_t N = size_t(1) << a.n;
	int32_t *r = a.desc[t].regs + static_cast<size_t>(a.dst) * N;
	for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < N; i += size_t(gridDim.x) * blockDim.x)
		r[i] = (i == 0) ? value : 0;
}

// reg[dst] = reg[src] for every test of the launch.
__global__ void k_copy(const Args a)
{
	const int t = a.tests[blockIdx.y];
	const size_t N = size_t(1) << a.n;
	const int4 *s = reinterpret_cast<const int4 *>(a.desc[t].regs + static_cast<size_t>(a.src) * N);
	int4 *o = reinterpret_cast<int4 *>(a.desc[t].regs + static_cast<size_t>(a.dst) * N);
	for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < N / 4; i += size_t(gridDim.x) * blockDim.x)
		o[i] = s[i];
}

// pos[t] = max(pos[t] - count, -1) for every test (end of a four-step block;
// k_small advances its own tests the same way).
__global__ void k_pos_sub(int64_t *pos, const int32_t *tests, int ntests, int count)
{
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i < ntests)
	{
		const int64_t p = pos[tests[i]] - count;
		pos[tests[i]] = (p < -1) ? -1 : p;
	}
}

}  // namespace gfc
