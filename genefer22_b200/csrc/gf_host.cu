// gf_host.cu -- host runtime and C ABI of the B200 modular-squaring engine.
//
// Owns device memory, root tables, kernel plans and CUDA graphs, and
// implements include/gfcuda.h.  The single-test calls mirror genefer's
// `transform` interface (src/transform.h:42-256); the batch calls run many
// tests of one size class per launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/gfcuda.h"
#include "gf_kernels.cuh"

using namespace gfc;

namespace {

thread_local std::string g_err;
std::atomic<uint64_t> g_launches{0};

struct Error
{
	int code;
	std::string msg;
};

[[noreturn]] void fail(int code, const std::string &msg) { throw Error{code, msg}; }

#define GFC_CK(x)                                                                                     \
	do                                                                                                \
	{                                                                                                 \
		const cudaError_t e_ = (x);                                                                   \
		if (e_ != cudaSuccess) fail(GFC_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_));   \
	} while (0)

inline void after_launch()
{
	g_launches.fetch_add(1, std::memory_order_relaxed);
	const cudaError_t e = cudaGetLastError();
	if (e != cudaSuccess) fail(GFC_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
}

// kernel<<<grid, block, smem, s>>>(a) with programmatic stream serialization:
// the grid may be scheduled while the previous kernel of the stream drains,
// and waits at its start (pdl_wait) until that kernel has completed, so memory
// effects keep the order of plain launches while the launch and ramp-up
// overlap the previous kernel's tail (one squaring per call at n = 16, 17:
// +38 %, +41 % measured on one B200).  Under stream capture only when
// a.pdl_graph is set: graph replays with programmatic edges measured 2-4 %
// faster for packed plans with middle passes of at most 2^5 points
// (n = 17..22) and up to 9 % slower for others (unpacked n = 13, 14; plan 306).
template <class K>
void launch_pdl(K *kernel, dim3 grid, dim3 block, size_t smem, cudaStream_t s, const Args &a)
{
	cudaLaunchConfig_t cfg = {};
	cfg.gridDim = grid;
	cfg.blockDim = block;
	cfg.dynamicSmemBytes = smem;
	cfg.stream = s;
	cudaLaunchAttribute at[1];
	at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
	at[0].val.programmaticStreamSerializationAllowed = 1;
	cfg.attrs = at;
	cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
	GFC_CK(cudaStreamIsCapturing(s, &cs));
	cfg.numAttrs = ((cs == cudaStreamCaptureStatusNone) || (a.pdl_graph != 0)) ? 1 : 0;
	GFC_CK(cudaLaunchKernelEx(&cfg, kernel, a));
	after_launch();
}

// ------------------------------------------------------------------ roots

// Prime slots: set 0 = slots 0,1; set 1 = slots 2,3,4.
const uint32_t kPrime[5] = { PrimeSet<0>::p[0], PrimeSet<0>::p[1], PrimeSet<1>::p[0], PrimeSet<1>::p[1], PrimeSet<1>::p[2] };

inline uint32_t mulmod_h(uint32_t a, uint32_t b, uint32_t p) { return static_cast<uint32_t>((static_cast<uint64_t>(a) * b) % p); }

uint32_t powmod_h(uint32_t a, uint64_t e, uint32_t p)
{
	uint32_t r = 1, y = a % p;
	while (e != 0) { if (e & 1) r = mulmod_h(r, y, p); y = mulmod_h(y, y, p); e >>= 1; }
	return r;
}

// Smallest generator of (Z/pZ)*: g^((p-1)/q) != 1 for every prime q | p-1.
uint32_t primitive_root(uint32_t p)
{
	std::vector<uint32_t> f;
	uint32_t m = p - 1;
	for (uint32_t q = 2; static_cast<uint64_t>(q) * q <= m; ++q)
		if (m % q == 0) { f.push_back(q); while (m % q == 0) m /= q; }
	if (m > 1) f.push_back(m);
	for (uint32_t g = 2;; ++g)
	{
		bool ok = true;
		for (uint32_t q : f) if (powmod_h(g, (p - 1) / q, p) == 1) { ok = false; break; }
		if (ok) return g;
	}
}

inline uint32_t to_mont_h(uint32_t x, uint32_t p) { return static_cast<uint32_t>((static_cast<uint64_t>(x % p) << 32) % p); }

inline uint32_t bitrev(uint32_t k, int n)
{
	uint32_t r = 0;
	for (int i = 0; i < n; ++i) { r = (r << 1) | (k & 1); k >>= 1; }
	return r;
}

// Words per table entry: the 31-bit primes keep each root with its Shoup
// quotient (gf_arith.cuh, RootS), the 32-bit primes one Montgomery word.
inline size_t root_words(uint32_t p) { return (p < (1u << 31)) ? 2 : 1; }

// Entry k of a root table: psi^e in Montgomery form (32-bit primes), or in
// normal form followed by floor(w 2^32 / p) (31-bit primes).
inline void put_root(uint32_t *t, size_t k, uint32_t w, uint32_t p)
{
	if (root_words(p) == 1) { t[k] = to_mont_h(w, p); return; }
	t[2 * k] = w;
	t[2 * k + 1] = static_cast<uint32_t>((static_cast<uint64_t>(w) << 32) / p);
}

// Root tables of one prime for length N = 2^n (N entries of root_words(p)
// words; layout in gf_ntt.cuh), built on the device (k_roots):
//   entry k of fw = psi^bitrev_n(k), of iv = psi^-bitrev_n(k)  (k >= 1),
//   word 0 of fw = R^2 / N (normalisation c), of iv = psi^(-N/2) c (k0), in
//   Montgomery form (R = 2^32).
// The host finds psi and the entry-0 constants; the kernel writes the N
// entries of both tables with one product per entry.  fw and iv are device
// pointers; `s` a stream of the device.
void build_roots_device(uint32_t p, int n, uint32_t *fw, uint32_t *iv, cudaStream_t s, bool packed = false)
{
	const uint32_t N = 1u << n;
	const uint32_t psi = powmod_h(primitive_root(p), (p - 1) / (2ull * N), p);
	if (powmod_h(psi, N, p) != p - 1) fail(GFC_ERR_ARG, "root table: psi is not a primitive 2N-th root");
	const uint32_t psi_inv = powmod_h(psi, 2ull * N - 1, p);
	const uint32_t R1 = static_cast<uint32_t>((uint64_t(1) << 32) % p);
	const uint32_t c = mulmod_h(mulmod_h(R1, R1, p), powmod_h(N % p, p - 2, p), p);
	const uint32_t k0 = mulmod_h(p - powmod_h(psi, N / 2, p), c, p);
	// word 1 of entry 0 (31-bit primes): for inputs packed as D 2^-32
	// (pack_residue, the packed tables' 8-row columns), 2^64 more on the square
	const uint32_t c2 = packed ? mulmod_h(c, mulmod_h(R1, R1, p), p) : 0u;
	const uint32_t k02 = packed ? mulmod_h(p - powmod_h(psi, N / 2, p), c2, p) : 0u;
	const int run = 64, threads = 256;
	const uint32_t runs = (N + run - 1) / run;
	k_roots<<<(runs + threads - 1) / threads, threads, 0, s>>>(fw, iv, p, psi, psi_inv, n, static_cast<int>(root_words(p)),
															   run, c, k0, c2, k02);
	const cudaError_t e = cudaGetLastError();
	if (e != cudaSuccess) fail(GFC_ERR_CUDA, std::string("root table kernel: ") + cudaGetErrorString(e));
}

// ------------------------------------------------------------------ memory
//
// Device memory of batches and root tables comes from a stream-ordered pool
// per device and goes back with cudaFreeAsync; pinned staging comes from a
// cache of page-locked chunks.  cudaFree and cudaFreeHost wait for the whole
// device, so a batch closed by one thread while others ran held every
// thread's CUDA calls behind the work in flight on all streams, and pinning
// fresh pages is slow.  Both keep freed memory for reuse up to a retention
// limit: none by default, a server's budget while one runs.
struct MemState
{
	std::mutex mu;
	std::map<int, cudaMemPool_t> pools;
	std::map<int, cudaStream_t> release;          // per device: frees of memory no work uses
	std::map<void *, size_t> pinned;              // every live pinned chunk with its size
	std::multimap<size_t, void *> pinned_free;    // cached chunks by size
	size_t pinned_cached = 0;
	size_t retain = 0;                            // bytes kept per device pool and in the pinned cache
	int retainers = 0;
};

// Never destroyed: the CUDA runtime may be gone when static objects die.
MemState &mem_state()
{
	static MemState *m = new MemState();
	return *m;
}

size_t pinned_cap(const MemState &m) { return std::min(m.retain, size_t(32) << 30); }

// The pool of the current device `device` (created on first use).
cudaMemPool_t dev_pool(int device)
{
	MemState &m = mem_state();
	std::lock_guard<std::mutex> l(m.mu);
	auto it = m.pools.find(device);
	if (it != m.pools.end()) return it->second;
	cudaMemPoolProps pp{};
	pp.allocType = cudaMemAllocationTypePinned;
	pp.handleTypes = cudaMemHandleTypeNone;
	pp.location.type = cudaMemLocationTypeDevice;
	pp.location.id = device;
	cudaMemPool_t pool = nullptr;
	GFC_CK(cudaMemPoolCreate(&pool, &pp));
	uint64_t keep = m.retain;
	GFC_CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
	cudaStream_t rs = nullptr;
	GFC_CK(cudaStreamCreateWithFlags(&rs, cudaStreamNonBlocking));
	m.pools[device] = pool;
	m.release[device] = rs;
	return pool;
}

// Device memory ordered on stream s (usable elsewhere once s has synchronised).
void *dev_alloc(int device, size_t bytes, cudaStream_t s)
{
	void *p = nullptr;
	GFC_CK(cudaMallocFromPoolAsync(&p, bytes, dev_pool(device), s));
	return p;
}

// Returns memory of dev_alloc that no queued or running work uses any more.
void dev_free(int device, void *p)
{
	if (p == nullptr) return;
	cudaStream_t rs = nullptr;
	{
		MemState &m = mem_state();
		std::lock_guard<std::mutex> l(m.mu);
		auto it = m.release.find(device);
		if (it != m.release.end()) rs = it->second;
	}
	if (rs != nullptr) cudaFreeAsync(p, rs);
}

// Page-locked host memory of at least `bytes` (nullptr when CUDA refuses).
void *pinned_get(size_t bytes)
{
	bytes = (bytes + 65535) & ~size_t(65535);
	MemState &m = mem_state();
	{
		std::lock_guard<std::mutex> l(m.mu);
		auto it = m.pinned_free.lower_bound(bytes);
		if ((it != m.pinned_free.end()) && (it->first <= 2 * bytes))
		{
			void *p = it->second;
			m.pinned_cached -= it->first;
			m.pinned_free.erase(it);
			return p;
		}
	}
	void *p = nullptr;
	if (cudaHostAlloc(&p, bytes, cudaHostAllocPortable) != cudaSuccess)
	{
		(void)cudaGetLastError();
		return nullptr;
	}
	std::lock_guard<std::mutex> l(m.mu);
	m.pinned[p] = bytes;
	return p;
}

// Memory of pinned_get whose copies have all completed.
void pinned_put(void *p)
{
	if (p == nullptr) return;
	MemState &m = mem_state();
	{
		std::lock_guard<std::mutex> l(m.mu);
		auto it = m.pinned.find(p);
		if (it == m.pinned.end()) return;
		if (m.pinned_cached + it->second <= pinned_cap(m))
		{
			m.pinned_free.emplace(it->second, p);
			m.pinned_cached += it->second;
			return;
		}
		m.pinned.erase(it);
	}
	cudaFreeHost(p);
}

// A private stream for building tables, synchronised and destroyed on scope exit.
struct TableStream
{
	cudaStream_t s = nullptr;
	TableStream() { GFC_CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)); }
	~TableStream() { if (s != nullptr) cudaStreamDestroy(s); }
	void sync() { GFC_CK(cudaStreamSynchronize(s)); }
};

// Twist factors of one six-step split (k_twist) for every prime of a table.
struct TwistTables
{
	uint32_t *d = nullptr;
	const uint32_t *tf[3][4] = {}, *ti[3][4] = {};
};

struct DeviceTables
{
	int device = -1, n = 0;
	uint32_t *d = nullptr;
	Tables tab[3];
	std::mutex tw_mu;
	std::map<int, TwistTables> twist;   // by log2 rows of the split, built on first use
	// every holder synchronised its stream before letting go of the tables
	~DeviceTables()
	{
		for (auto &t : twist) dev_free(device, t.second.d);
		dev_free(device, d);
	}
};

std::mutex g_tab_mu;
std::map<std::pair<int, int>, std::weak_ptr<DeviceTables>> g_tab_cache;

// Root tables for (device, n), shared by every handle of that size.
std::shared_ptr<DeviceTables> get_tables(int device, int n)
{
	std::lock_guard<std::mutex> lock(g_tab_mu);
	const auto key = std::make_pair(device, n);
	auto it = g_tab_cache.find(key);
	if (it != g_tab_cache.end())
		if (auto sp = it->second.lock()) return sp;

	auto t = std::make_shared<DeviceTables>();
	t->device = device; t->n = n;
	const size_t N = size_t(1) << n;
	size_t off[5], total = 0;
	for (int s = 0; s < 5; ++s) { off[s] = total; total += 2 * root_words(kPrime[s]) * N; }
	{
		TableStream ts;
		t->d = static_cast<uint32_t *>(dev_alloc(device, total * sizeof(uint32_t), ts.s));
		for (int s = 0; s < 5; ++s)
		{
			const size_t words = root_words(kPrime[s]) * N;
			build_roots_device(kPrime[s], n, t->d + off[s], t->d + off[s] + words, ts.s);
		}
		ts.sync();
	}
	const int slot0[2] = { 0, 2 };
	for (int set = 0; set < 2; ++set)
		for (int pl = 0; pl < 3; ++pl)
		{
			const int s = (set == 0 && pl == 2) ? 1 : slot0[set] + pl;   // set 0 has 2 planes; plane 2 unused
			t->tab[set].fw[pl] = t->d + off[s];
			t->tab[set].iv[pl] = t->d + off[s] + root_words(kPrime[s]) * N;
		}
	g_tab_cache[key] = t;
	return t;
}

// The six-step twist factors of table t (2^t.n points, prime sets 0 and 1,
// or set 2 when `packed`) for R = 2^lr rows, built on the device on first use.
const TwistTables &get_twist(DeviceTables &t, bool packed, int lr)
{
	std::lock_guard<std::mutex> lock(t.tw_mu);
	auto it = t.twist.find(lr);
	if (it != t.twist.end()) return it->second;
	const int n = t.n;
	const size_t C = size_t(1) << (n - lr);
	uint32_t primes[5];
	int np = 0;
	if (packed) for (int pl = 0; pl < 4; ++pl) primes[np++] = PrimeSet<2>::p[pl];
	else for (int s = 0; s < 5; ++s) primes[np++] = kPrime[s];
	size_t off[5], total = 0;
	for (int k = 0; k < np; ++k) { off[k] = total; total += 2 * (16 + root_words(primes[k])) * C; }
	TwistTables tw;
	{
		TableStream ts;
		tw.d = static_cast<uint32_t *>(dev_alloc(t.device, total * sizeof(uint32_t), ts.s));
		for (int k = 0; k < np; ++k)
		{
			const uint32_t p = primes[k], N = 1u << n;
			const uint32_t psi = powmod_h(primitive_root(p), (p - 1) / (2ull * N), p);
			const uint32_t psi_inv = powmod_h(psi, 2ull * N - 1, p);
			const size_t words = (16 + root_words(p)) * C;
			const unsigned blocks = static_cast<unsigned>((16 * C + 255) / 256);
			k_twist<<<blocks, 256, 0, ts.s>>>(tw.d + off[k], tw.d + off[k] + words, p, psi, psi_inv, n, lr,
											  static_cast<int>(root_words(p)));
			const cudaError_t e = cudaGetLastError();
			if (e != cudaSuccess)
			{
				ts.sync();
				dev_free(t.device, tw.d);
				fail(GFC_ERR_CUDA, std::string("twist table kernel: ") + cudaGetErrorString(e));
			}
		}
		ts.sync();
	}
	for (int k = 0; k < np; ++k)
	{
		const size_t words = (16 + root_words(primes[k])) * C;
		const int set = packed ? 2 : ((k < 2) ? 0 : 1), pl = packed ? k : ((k < 2) ? k : k - 2);
		tw.tf[set][pl] = tw.d + off[k];
		tw.ti[set][pl] = tw.d + off[k] + words;
	}
	if (!packed)
	{
		// set 0 has two planes; its plane 2 is unused (as in the root tables)
		tw.tf[0][2] = tw.tf[0][1];
		tw.ti[0][2] = tw.ti[0][1];
	}
	return t.twist.emplace(lr, tw).first->second;
}

// Exact range: with |digit| <= D = b/2 + 1 every coefficient of a product of
// two resting registers is at most N D^2 in absolute value; the centred CRT
// of set S is exact when N D^2 < floor(M_S / 2).
int choose_set(uint32_t b, int n)
{
	const u128 D = b / 2 + 1;
	const u128 bound = (u128(1) << n) * D * D;
	const u128 M0 = u128(PrimeSet<0>::p[0]) * PrimeSet<0>::p[1];
	const u128 M1 = u128(PrimeSet<1>::p[0]) * PrimeSet<1>::p[1] * PrimeSet<1>::p[2];
	if (bound < M0 / 2) return 0;
	if (bound < M1 / 2) return 1;
	return -1;
}

// Root tables of prime set 2 for the packed transform of 2^np points
// (cached under key -np).
std::shared_ptr<DeviceTables> get_tables_packed(int device, int np)
{
	std::lock_guard<std::mutex> lock(g_tab_mu);
	const auto key = std::make_pair(device, -np);
	auto it = g_tab_cache.find(key);
	if (it != g_tab_cache.end())
		if (auto sp = it->second.lock()) return sp;
	auto t = std::make_shared<DeviceTables>();
	t->device = device; t->n = np;
	const size_t N = size_t(1) << np;
	const size_t words = 2 * N;                       // 31-bit primes: root and Shoup quotient
	{
		TableStream ts;
		t->d = static_cast<uint32_t *>(dev_alloc(device, 8 * words * sizeof(uint32_t), ts.s));
		for (int pl = 0; pl < 4; ++pl)
		{
			t->tab[2].fw[pl] = t->d + (2 * pl) * words;
			t->tab[2].iv[pl] = t->d + (2 * pl + 1) * words;
			build_roots_device(PrimeSet<2>::p[pl], np, t->d + (2 * pl) * words, t->d + (2 * pl + 1) * words, ts.s, true);
		}
		ts.sync();
	}
	g_tab_cache[key] = t;
	return t;
}

// Packed digits (two base-b digits per coefficient, prime set 2) are exact
// when every coefficient of the half-length product, at most
// (N/2) ((b/2 + 1)(b + 1))^2, is below floor(M_2 / 2); the limb split of the
// CRT value wants 2^20 <= b < 2^28.
bool packed_ok(uint32_t b, int n)
{
	if ((b < (1u << 20)) || (b >= (1u << 28))) return false;
	const u128 D = u128(b / 2 + 1) * (u128(b) + 1);
	const u128 M2 = u128(PrimeSet<2>::p[0]) * PrimeSet<2>::p[1] * PrimeSet<2>::p[2] * PrimeSet<2>::p[3];
	return D * D < (M2 / 2) / (u128(1) << (n - 1));
}

void base_limbs(u128 w, uint32_t b, uint32_t *out, int count)
{
	for (int j = 0; j < count; ++j) { out[j] = static_cast<uint32_t>(w % b); w /= b; }
	if (w != 0) fail(GFC_ERR_RANGE, "packed digits: weight does not fit its limbs");
}

PackK pack_constants(uint32_t b)
{
	PackK P{};
	const u128 p1 = PrimeSet<2>::p[0], p2 = PrimeSet<2>::p[1], p3 = PrimeSet<2>::p[2];
	for (int f = 1; f <= 2; ++f)
	{
		base_limbs(f * p1, b, P.w1[f - 1], 2);
		base_limbs(f * p1 * p2, b, P.w2[f - 1], 4);
		base_limbs(f * p1 * p2 * p3, b, P.w3[f - 1], 5);
	}
	for (int k = 0; k < 4; ++k)
	{
		const uint32_t p = PrimeSet<2>::p[k];
		P.bm[k] = static_cast<uint32_t>((static_cast<uint64_t>(b % p) << 32) % p);
	}
	return P;
}

// Constants of the fused CRT + carry (gf_arith.cuh, CarryK) for base b.
CarryK carry_constants(uint32_t b, int set)
{
	const u128 T = (set == 0) ? u128(PrimeSet<0>::p[0]) : u128(PrimeSet<1>::p[0]) * PrimeSet<1>::p[1];
	const u128 M = (set == 0) ? u128(PrimeSet<0>::p[0]) * PrimeSet<0>::p[1]
							  : u128(PrimeSet<1>::p[0]) * PrimeSet<1>::p[1] * PrimeSet<1>::p[2];
	CarryK k{};
	k.b = b;
	k.h = b / 2;
	k.binv = ~uint64_t(0) / b;
	k.k = ((uint64_t(1) << 56) + b - 1) / b;
	k.kb = k.k * b;
	k.kw = ((uint64_t(1) << 62) + b - 1) / b;
	k.kwb = k.kw * b;
	for (int f = 1; f <= 2; ++f)
	{
		k.q[f - 1] = static_cast<uint64_t>((f * T) / b);
		k.r[f - 1] = static_cast<uint32_t>((f * T) % b);
		k.mq[f - 1] = static_cast<uint64_t>((f * M) / b);   // modulo 2^64
		k.mr[f - 1] = static_cast<uint32_t>((f * M) % b);
	}
	return k;
}

// ------------------------------------------------------------------ launch dispatch

constexpr int FIX_THREADS = 256;

template <class K>
void set_smem(K kernel, size_t smem)
{
	GFC_CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
}

// `prep` only raises the kernel's shared-memory limit (done outside graph capture).
// Streaming multiprocessors of the current device (cached per device).
int sm_count()
{
	static std::atomic<int> cache[64];
	int dev = 0;
	GFC_CK(cudaGetDevice(&dev));
	if ((dev < 0) || (dev >= 64)) return 148;
	int v = cache[dev].load();
	if (v == 0)
	{
		GFC_CK(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev));
		cache[dev].store(v);
	}
	return v;
}

template <int SET, int LOGN>
void small_t(const Args &a, int grid, cudaStream_t s, bool prep)
{
	using S = SmallShape<SET, LOGN, false>;
	using SS = SmallShape<SET, LOGN, true>;
	if (prep)
	{
		set_smem(k_small<SET, LOGN, false>, S::SMEM);
		set_smem(k_small<SET, LOGN, true>, SS::SMEM);
		return;
	}
	// fewer tests than SMs: plane-split passes (more warps per test)
	if (SS::PSPLIT && (grid < sm_count())) launch_pdl(k_small<SET, LOGN, true>, dim3(grid), dim3(SS::T), SS::SMEM, s, a);
	else launch_pdl(k_small<SET, LOGN, false>, dim3(grid), dim3(S::T), S::SMEM, s, a);
}

template <int SET>
void small_set(int logn, const Args &a, int grid, cudaStream_t s, bool prep)
{
	switch (logn)
	{
		case 10: small_t<SET, 10>(a, grid, s, prep); break;
		case 11: small_t<SET, 11>(a, grid, s, prep); break;
		case 12: small_t<SET, 12>(a, grid, s, prep); break;
		case 13: small_t<SET, 13>(a, grid, s, prep); break;
		case 14: small_t<SET, 14>(a, grid, s, prep); break;
		default: fail(GFC_ERR_ARG, "single-CTA plan needs 10 <= n <= 14");
	}
}

// A register column launch whose one-thread-per-column grid (256 columns and
// 8 warps per CTA) holds fewer than `per_sm` warps per SM takes the
// plane-split kernels instead: a thread per (plane, column).  Measured on one
// B200: the packed kernels gain below a full SM (32 warps); the unpacked ones,
// whose CRT phase keeps one thread per segment, only below 8 warps per SM.
bool split_cols(size_t cols, int grid_y, int per_sm)
{
	return (cols / 256) * static_cast<size_t>(grid_y) * 8 < static_cast<size_t>(sm_count()) * static_cast<size_t>(per_sm);
}

template <int LR>
void col_t(bool inv, const Args &a, int grid_y, cudaStream_t s, bool prep)
{
	if constexpr (LR <= 4)
	{
		// R <= 16: a thread owns a column (register kernels)
		using S = ColRegShape<LR>;
		if (prep) { set_smem(k_colr_inv<LR>, S::SMEM); return; }
		const size_t cols = size_t(1) << (a.n - LR);
		if (split_cols(cols, grid_y, 8))
		{
			const dim3 grid(static_cast<unsigned>(cols / CS_T), static_cast<unsigned>(grid_y));
			if (inv) launch_pdl(k_colr_inv_s<LR>, grid, dim3(WMAX * CS_T), 0, s, a);
			else launch_pdl(k_colr_fwd_s<LR>, grid, dim3(WMAX * CS_T), 0, s, a);
			return;
		}
		const dim3 grid(static_cast<unsigned>(cols / COLR_THREADS), static_cast<unsigned>(grid_y));
		if (inv) launch_pdl(k_colr_inv<LR>, grid, dim3(COLR_THREADS), S::SMEM, s, a);
		else launch_pdl(k_colr_fwd<LR>, grid, dim3(COLR_THREADS), 0, s, a);
	}
	else
	{
		using S = ColShape<LR>;
		if (prep) { set_smem(k_col_fwd<LR>, S::SMEM); set_smem(k_col_inv<LR>, S::SMEM); return; }
		const dim3 grid(static_cast<unsigned>((size_t(1) << (a.n - LR)) / S::CW), static_cast<unsigned>(grid_y));
		if (inv) launch_pdl(k_col_inv<LR>, grid, dim3(col_threads(LR)), S::SMEM, s, a);
		else launch_pdl(k_col_fwd<LR>, grid, dim3(col_threads(LR)), S::SMEM, s, a);
	}
}

void launch_col(int lr, bool inv, const Args &a, int grid_y, cudaStream_t s, bool prep)
{
	switch (lr)
	{
		case 3: col_t<3>(inv, a, grid_y, s, prep); break;
		case 4: col_t<4>(inv, a, grid_y, s, prep); break;
		case 5: col_t<5>(inv, a, grid_y, s, prep); break;
		case 6: col_t<6>(inv, a, grid_y, s, prep); break;
		case 7: col_t<7>(inv, a, grid_y, s, prep); break;
		case 8: col_t<8>(inv, a, grid_y, s, prep); break;
		case 9: col_t<9>(inv, a, grid_y, s, prep); break;
		case 10: col_t<10>(inv, a, grid_y, s, prep); break;
		default: fail(GFC_ERR_ARG, "four-step plan needs 3 <= lr <= 10");
	}
}

// Rows of 2^LC points, one (row, plane) per CTA; `planes` = 3, or 4 for
// packed digits (prime set 2).
template <int LC>
void row_t(const Args &a, int grid_y, cudaStream_t s, bool prep, int planes)
{
	using S = RowShape<LC>;
	const size_t smem = size_t(S::PC) * 4;          // one plane per CTA
	if (prep) { set_smem(k_row<LC>, smem); set_smem(k_row2<LC>, 2 * smem); set_smem(k_rowp<LC>, 2 * smem); return; }
	// A pair per CTA halves the grid: it pays for rows of 8192 points (512
	// threads, one CTA per SM) and from 1024 CTAs of single rows; below, the
	// single rows run in parallel instead (two packed tests at n = 17, 128 row
	// CTAs: 36.6 -> 22.5 us per squaring unpaired, four 42.4 -> 35.0; two at
	// n = 18 with 8192-point rows 37.2 paired against 39.6).
	const bool pair = (LC >= 13) || ((size_t(1) << (a.n - LC)) * 4 * size_t(grid_y) >= 1024);
	if ((planes == 4) && (a.op != OP_FWD) && a.twist && pair)
	{
		// twisted packed rows share their roots: two rows of a test per CTA (k_rowp)
		const dim3 grid((1u << (a.n - LC - 1)) * 4u, static_cast<unsigned>(grid_y));
		launch_pdl(k_rowp<LC>, grid, dim3(row_threads(LC)), 2 * smem, s, a);
		return;
	}
	if ((planes == 4) && (a.op != OP_FWD) && (grid_y >= 2) && pair)
	{
		// packed batches: two tests per CTA sharing the row's roots (k_row2)
		const dim3 grid((1u << (a.n - LC)) * 4u, static_cast<unsigned>((grid_y + 1) / 2));
		cudaLaunchConfig_t cfg = {};
		cfg.gridDim = grid;
		cfg.blockDim = dim3(row_threads(LC));
		cfg.dynamicSmemBytes = 2 * smem;
		cfg.stream = s;
		cudaLaunchAttribute at[1];
		at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
		at[0].val.programmaticStreamSerializationAllowed = 1;
		cfg.attrs = at;
		cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
		GFC_CK(cudaStreamIsCapturing(s, &cs));
		cfg.numAttrs = ((cs == cudaStreamCaptureStatusNone) || (a.pdl_graph != 0)) ? 1 : 0;
		GFC_CK(cudaLaunchKernelEx(&cfg, k_row2<LC>, a, grid_y));
		after_launch();
		return;
	}
	const dim3 grid((1u << (a.n - LC)) * static_cast<unsigned>(planes), static_cast<unsigned>(grid_y));
	launch_pdl(k_row<LC>, grid, dim3(row_threads(LC)), smem, s, a);
}

void launch_row(int lc, const Args &a, int grid_y, cudaStream_t s, bool prep, int planes = 3)
{
	switch (lc)
	{
		case 8: row_t<8>(a, grid_y, s, prep, planes); break;
		case 9: row_t<9>(a, grid_y, s, prep, planes); break;
		case 10: row_t<10>(a, grid_y, s, prep, planes); break;
		case 11: row_t<11>(a, grid_y, s, prep, planes); break;
		case 12: row_t<12>(a, grid_y, s, prep, planes); break;
		case 13: row_t<13>(a, grid_y, s, prep, planes); break;
		default: fail(GFC_ERR_ARG, "four-step plan needs 8 <= n - lr <= 13");
	}
}

// Packed column kernels (prime set 2), a.n = log2 of the packed length.
template <int LR>
void pcol_t(bool inv, const Args &a, int grid_y, cudaStream_t s, bool prep)
{
	using S = PColShape<LR>;
	if (prep) { set_smem(k_pcol_inv<LR>, S::SMEM); return; }
	const size_t cols = size_t(1) << (a.n - LR);
	if (split_cols(cols, grid_y, 32))
	{
		const dim3 grid(static_cast<unsigned>(cols / PCS_T), static_cast<unsigned>(grid_y));
		// from 1024 CTAs (more than a wave at six CTAs per SM) six CTAs per SM
		// at 40 registers, else four at 64: one packed test per squaring, graph
		// replay on one B200, n = 22 135.8 -> 131.9 us, n = 21 73.6 -> 72.7,
		// four tests at n = 19 64.9 -> 64.2; a smaller grid (one test at n = 20,
		// 512 CTAs) ran 43.2 -> 47.5 us with the 40-register form
		const bool hi = size_t(grid.x) * grid.y >= 1024;
		if (inv)
		{
			if (hi) launch_pdl(k_pcol_inv_s<LR, PCS_MINB_HI>, grid, dim3(4 * PCS_T), 0, s, a);
			else launch_pdl(k_pcol_inv_s<LR, PCS_MINB_LO>, grid, dim3(4 * PCS_T), 0, s, a);
		}
		else if (hi) launch_pdl(k_pcol_fwd_s<LR, PCS_MINB_HI>, grid, dim3(4 * PCS_T), 0, s, a);
		else launch_pdl(k_pcol_fwd_s<LR, PCS_MINB_LO>, grid, dim3(4 * PCS_T), 0, s, a);
		return;
	}
	const dim3 grid(static_cast<unsigned>(cols / PCOL_THREADS), static_cast<unsigned>(grid_y));
	if (inv) launch_pdl(k_pcol_inv<LR>, grid, dim3(PCOL_THREADS), S::SMEM, s, a);
	else launch_pdl(k_pcol_fwd<LR>, grid, dim3(PCOL_THREADS), 0, s, a);
}

void launch_pcol(int lr, bool inv, const Args &a, int grid_y, cudaStream_t s, bool prep)
{
	switch (lr)
	{
		case 3: pcol_t<3>(inv, a, grid_y, s, prep); break;
		case 4: pcol_t<4>(inv, a, grid_y, s, prep); break;
		default: fail(GFC_ERR_ARG, "packed plan needs lr = 3 or 4");
	}
}

// Cluster-resident squaring (k_cluster): `prep` raises the shared-memory limit,
// allows 16-CTA clusters and returns in *max_out how many clusters fit on the
// device at once; otherwise launches a persistent grid of
// min(ntests, max_active) clusters over the tests a.tests[0 .. ntests-1].
template <int LQ, int LC>
void cluster_t(const Args &a, int ntests, int max_active, cudaStream_t s, bool prep, int *max_out)
{
	using S = ClusterShape<LQ, LC>;
	auto kern = k_cluster<LQ, LC>;
	cudaLaunchConfig_t cfg = {};
	cudaLaunchAttribute at[1];
	at[0].id = cudaLaunchAttributeClusterDimension;
	at[0].val.clusterDim.x = S::Q; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
	cfg.blockDim = dim3(S::T);
	cfg.dynamicSmemBytes = S::SMEM;
	cfg.attrs = at; cfg.numAttrs = 1;
	if (prep)
	{
		set_smem(kern, S::SMEM);
		if (S::Q > 8) GFC_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
		cfg.gridDim = dim3(S::Q);
		int m = 0;
		GFC_CK(cudaOccupancyMaxActiveClusters(&m, kern, &cfg));
		if (m < 1) fail(GFC_ERR_CUDA, "cluster plan: no cluster of this size fits on the device");
		*max_out = m;
		return;
	}
	const int ncl = (ntests < max_active) ? ntests : max_active;
	cfg.gridDim = dim3(static_cast<unsigned>(ncl * S::Q));
	cfg.stream = s;
	// programmatic stream serialization as launch_pdl: the clusters start when
	// the previous kernel of the stream has completed (pdl_wait), its launch overlapping that kernel's tail
	cudaLaunchAttribute at2[2] = { at[0], {} };
	at2[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
	at2[1].val.programmaticStreamSerializationAllowed = 1;
	cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
	GFC_CK(cudaStreamIsCapturing(s, &cs));
	cfg.attrs = at2;
	cfg.numAttrs = (cs == cudaStreamCaptureStatusNone) ? 2 : 1;
	GFC_CK(cudaLaunchKernelEx(&cfg, kern, a, ntests));
	after_launch();
}

// Cluster shape by size: n = 12..14 with plane-split passes on rows of
// 2^(n-LQ) (eight CTAs at n = 12, 16 at n = 13, 14), n = 15..17 on 2..16 CTAs
// with rows of 2^13.  One test on one B200 (graph replay, us per squaring),
// 8 -> 16 CTAs with the balanced row schedule: n = 12 6.75 -> 9.95 (2^8-point
// rows of two 16-point passes leave half of the threads idle), n = 13 8.80 ->
// 8.31; n = 14 13.04 (eight CTAs, earlier schedule) -> 10.40.
void launch_cluster_n(int n, const Args &a, int ntests, int max_active, cudaStream_t s, bool prep, int *max_out)
{
	switch (n)
	{
		case 12: cluster_t<3, 9>(a, ntests, max_active, s, prep, max_out); break;
		case 13: cluster_t<4, 9>(a, ntests, max_active, s, prep, max_out); break;
		case 14: cluster_t<4, 10>(a, ntests, max_active, s, prep, max_out); break;
		case 15: cluster_t<2, 13>(a, ntests, max_active, s, prep, max_out); break;
		case 16: cluster_t<3, 13>(a, ntests, max_active, s, prep, max_out); break;
		case 17: cluster_t<4, 13>(a, ntests, max_active, s, prep, max_out); break;
		default: fail(GFC_ERR_ARG, "cluster plan needs 12 <= n <= 17");
	}
}

// Six-step middle pass (k_mid): planes of every test, tiles of 2^lr2 rows.
template <int LR2>
void mid_t(bool inv, const Args &a, int grid_y, cudaStream_t s, bool prep, int planes)
{
	using S = MidShape<LR2>;
	const size_t smem = size_t(planes) * S::PS * 4;
	if (prep)
	{
		set_smem(k_mid<LR2, false>, S::SMEM);
		set_smem(k_mid<LR2, true>, S::SMEM);
		return;
	}
	const size_t C = size_t(1) << (a.n - MID_LR1 - LR2);
	const dim3 grid(static_cast<unsigned>((size_t(1) << MID_LR1) * (C / S::CW)), static_cast<unsigned>(grid_y));
	if (inv) launch_pdl(k_mid<LR2, true>, grid, dim3(col_threads(LR2)), smem, s, a);
	else launch_pdl(k_mid<LR2, false>, grid, dim3(col_threads(LR2)), smem, s, a);
}

// The middle pass in registers (k_midr): one thread per column of each plane.
template <int LR2>
void midr_t(bool inv, const Args &a, int grid_y, cudaStream_t s, bool prep, int planes)
{
	if (prep) return;
	const size_t C = size_t(1) << (a.n - MID_LR1 - LR2);
	const dim3 grid(static_cast<unsigned>((size_t(1) << MID_LR1) * size_t(planes) * (C / MIDR_THREADS)),
					static_cast<unsigned>(grid_y));
	if (inv) launch_pdl(k_midr<LR2, true>, grid, dim3(MIDR_THREADS), 0, s, a);
	else launch_pdl(k_midr<LR2, false>, grid, dim3(MIDR_THREADS), 0, s, a);
}

void launch_mid(int lr2, bool inv, const Args &a, int grid_y, cudaStream_t s, bool prep, int planes = 3)
{
	switch (lr2)
	{
		case 3: midr_t<3>(inv, a, grid_y, s, prep, planes); break;
		case 4: midr_t<4>(inv, a, grid_y, s, prep, planes); break;
		case 5: midr_t<5>(inv, a, grid_y, s, prep, planes); break;
		case 6:
		{
			// 64-point columns on thread pairs (k_midp): 128 registers, four CTAs per SM
			if (prep) break;
			const size_t C = size_t(1) << (a.n - MID_LR1 - 6);
			const dim3 grid(static_cast<unsigned>((size_t(1) << MID_LR1) * size_t(planes) * (C / MIDP_COLS)),
							static_cast<unsigned>(grid_y));
			if (inv) launch_pdl(k_midp<true>, grid, dim3(MIDP_THREADS), 0, s, a);
			else launch_pdl(k_midp<false>, grid, dim3(MIDP_THREADS), 0, s, a);
			break;
		}
		case 7: mid_t<7>(inv, a, grid_y, s, prep, planes); break;
		default: fail(GFC_ERR_ARG, "six-step plan needs 3 <= lr2 <= 7");
	}
}

constexpr int PLAN_SIX = 100;     // plan codes 100 + lr2: six-step, 2^4 x 2^lr2 column split
constexpr int PLAN_PACKED = 200;  // plan codes 200 + lr: packed digits, four-step of n - 1 with lr = 3, 4
constexpr int PLAN_PACKED_SIX = 300;   // plan codes 300 + lr2: packed digits, six-step of n - 1

constexpr int PLAN_CLUSTER = 1;   // plan code of the cluster-resident squaring
// A batch of at most this many tests of size 12..14 squares on the cluster
// plan by default: one test on 8 or 16 SMs instead of one (a lone n = 12, 13,
// 14 test on one CTA 15.4, 31.3, 62.4 us per squaring; on the cluster now
// 6.6, 8.2, 10.3, graph replay on one B200); larger batches fill the SMs with
// one CTA per test.
constexpr size_t CLUSTER_MAX_TESTS = 4;

bool plan_valid(int n, int lr)
{
	if (lr > PLAN_PACKED_SIX)
	{
		const int lr2 = lr - PLAN_PACKED_SIX, lc = n - 1 - MID_LR1 - lr2;
		return (lr2 >= 3) && (lr2 <= 7) && (lc >= 8) && (lc <= 13) && (col_width(lr2) <= (1 << lc));
	}
	if (lr > PLAN_PACKED)
	{
		const int l = lr - PLAN_PACKED, lc = n - 1 - l;
		return (l >= 3) && (l <= 4) && (lc >= 8) && (lc <= 13);
	}
	if (lr == PLAN_CLUSTER) return (n >= 12) && (n <= 17);
	if (lr > PLAN_SIX)
	{
		const int lr2 = lr - PLAN_SIX, lc = n - MID_LR1 - lr2;
		return (lr2 >= 3) && (lr2 <= 7) && (lc >= 8) && (lc <= 13) && (col_width(lr2) <= (1 << lc));
	}
	if (lr == 0) return (n >= 10) && (n <= SMALL_MAX_LOGN);
	const int lc = n - lr;
	return (lr >= 3) && (lr <= 10) && (lc >= 8) && (lc <= 13) && ((lr <= 4) || (col_width(lr) <= (1 << lc)));
}

// Default plans, the fastest per n measured on one B200 (graph replay of each
// candidate).  Without packed digits (single tests of 2 and 3 primes):
// single-CTA up to n = 14, four-step with rows of 2^12 at n = 15, 16, then
// six-step (16-point register column pass, register middle pass of 2^lr2
// points) with lr2 = 3 for n = 17, 18, 4 for n = 19, 20, 5 for n = 21, 6 for
// n = 22 and 7 for n = 23.
int default_plan(int n)
{
	if (n <= SMALL_MAX_LOGN) return 0;
	if (n <= 16) return n - 12;
	static const int lr2[24] = { 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 3, 3, 4, 4, 5, 6, 7 };
	return PLAN_SIX + lr2[n];
}

// The default packs a batch of at least this many tests whose bases all fit
// (0: never): packed digits are faster from one test at n >= 16 (measured on
// one B200 against the fastest unpacked plan).
size_t packed_min_tests(int n)
{
	// a lone n = 19 test: the unpacked six-step 104 (35.5 us per squaring) beats
	// the packed 303 (39.4 us) since the 64-point middle pass runs on thread pairs
	if (n == 19) return 2;
	return (n >= 16) ? 1 : 0;
}

// Default packed plan: four-step on N/2 with 8-row columns at n = 16 and
// 16-row columns at n = 17, 18; six-step on N/2 above.
int default_packed_plan(int n, size_t count)
{
	if (n == 16) return PLAN_PACKED + 3;
	if (n <= 18) return PLAN_PACKED + 4;
	// batches of two or more: 304 at n = 20, 21 and 306 at n = 22 (two tests, graph
	// replay on one B200: 66.6 -> 63.2, 126.1 -> 123.5, 242.5 -> 238.5 us per squaring)
	static const int lr2[24] = { 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 3, 3, 5, 5, 6 };
	static const int lr2_many[24] = { 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 3, 4, 4, 6, 6 };
	return PLAN_PACKED_SIX + ((count >= 2) ? lr2_many[n] : lr2[n]);
}

}  // namespace

// ------------------------------------------------------------------ batch object

struct gfc_batch
{
	int device = 0;
	cudaStream_t stream = nullptr;
	bool own_stream = false;
	int n = 0;
	size_t N = 0, count = 0, num_regs = 0;
	std::vector<uint32_t> b;
	std::vector<int> set;
	int lr = 0;
	std::shared_ptr<DeviceTables> tab;
	void *mem = nullptr;
	size_t mem_bytes = 0;
	int32_t *regs = nullptr;
	uint32_t *planes = nullptr, *zp = nullptr;
	int64_t *carry = nullptr, *d_pos = nullptr;
	TestDesc *d_desc = nullptr;
	int32_t *d_tests = nullptr;
	uint32_t *d_err = nullptr;
	std::vector<TestDesc> h_desc;
	std::vector<uint32_t *> ebits;
	int nset[2] = { 0, 0 }, offset[2] = { 0, 0 };   // tests per prime set; d_tests lists set 0 first
	int pending = -1;             // register whose segment carries are not yet absorbed (four-step)
	uint64_t sets_version = 0;    // bumped when a test changes prime set (per-set launches change)
	bool tests_sorted = true;     // d_tests lists the tests by prime set (only the single-CTA plan needs it)
	int cluster = 0;              // 1 when squarings use k_cluster (shape by n), else 0
	int six = 0;                  // lr2 of a six-step plan (columns 2^4 x 2^lr2, lr = 4 + lr2), else 0
	bool packed = false;          // prime set 2, two digits per coefficient, transform of N/2 (lr of that)
	std::shared_ptr<DeviceTables> tabp;   // root tables of prime set 2 at length N/2
	const TwistTables *twist = nullptr;   // six-step plans whose middle pass twists (lr2 <= 6)
	int cluster_max = 0;          // clusters of k_cluster resident at once
	bool capturing = false;
	uint64_t capture_start = 0;   // launch counter at capture_begin
	// Reserved slots (gfc_batch_reserve): exponent words of every slot in one
	// device buffer, and pinned host staging so that admission and the
	// asynchronous register copies allocate nothing and never synchronise.
	uint64_t res_bits = 0;        // exponent bits each slot can hold (0: not reserved)
	size_t res_words = 0;         // device words per slot
	uint32_t *d_eres = nullptr;   // count x res_words exponent words
	char *h_pin = nullptr;        // pinned: per slot [TestDesc | int64 pos | res_words words], then tests[], one
	size_t pin_slot = 0;          // bytes per slot in h_pin
	std::vector<cudaEvent_t> slot_ev;   // recorded after a slot's staged copies were enqueued

	// Waits for this batch's own stream only (not the device), then hands
	// its memory and its hold on the root tables back.
	~gfc_batch()
	{
		cudaSetDevice(device);
		if (stream != nullptr) cudaStreamSynchronize(stream);
		for (cudaEvent_t e : slot_ev) if (e != nullptr) cudaEventDestroy(e);
		dev_free(device, d_eres);
		pinned_put(h_pin);
		for (uint32_t *e : ebits) dev_free(device, e);
		dev_free(device, mem);
		if (own_stream && (stream != nullptr)) cudaStreamDestroy(stream);
	}
};

struct gfc_graph
{
	gfc_batch *batch = nullptr;
	int device = 0;
	cudaStream_t stream = nullptr;
	cudaGraph_t graph = nullptr;
	cudaGraphExec_t exec = nullptr;
	uint64_t kernels = 0;         // kernel nodes recorded
	uint64_t sets_version = 0;    // batch's sets_version at capture
	bool per_set = false;         // recorded per-prime-set launches (single-CTA plan)
	~gfc_graph()
	{
		cudaSetDevice(device);
		if (exec != nullptr) cudaGraphExecDestroy(exec);
		if (graph != nullptr) cudaGraphDestroy(graph);
	}
};

namespace {

// Switches every test's descriptor between its own prime set (0 or 1, digits
// one per coefficient) and prime set 2 (packed digits).
void set_packed(gfc_batch &bt, bool on)
{
	for (size_t i = 0; i < bt.count; ++i)
	{
		TestDesc &d = bt.h_desc[i];
		if (on)
		{
			d.set = 2;
			d.ck = carry_constants(bt.b[i], 1);
			d.pk = pack_constants(bt.b[i]);
		}
		else
		{
			d.set = bt.set[i];
			d.ck = carry_constants(bt.b[i], bt.set[i]);
		}
	}
	if (on) bt.tabp = get_tables_packed(bt.device, bt.n - 1);
	GFC_CK(cudaMemcpy(bt.d_desc, bt.h_desc.data(), bt.count * sizeof(TestDesc), cudaMemcpyHostToDevice));
}

// Sets the batch's kernels from a plan code (see gfc_batch_set_plan).
void apply_plan(gfc_batch &bt, int code)
{
	bt.cluster = 0;
	bt.six = 0;
	bt.packed = false;
	if (code > PLAN_PACKED_SIX)
	{
		bt.packed = true;
		bt.six = code - PLAN_PACKED_SIX;
		bt.lr = MID_LR1 + bt.six;
	}
	else if (code > PLAN_PACKED)
	{
		bt.packed = true;
		bt.lr = code - PLAN_PACKED;
	}
	else if (code == PLAN_CLUSTER)
	{
		// products keep the default plan of 15 <= n <= 17
		apply_plan(bt, default_plan(bt.n));
		bt.cluster = 1;
	}
	else if (code > PLAN_SIX)
	{
		bt.six = code - PLAN_SIX;
		bt.lr = MID_LR1 + bt.six;
	}
	else bt.lr = code;
}

void check_reg(const gfc_batch &bt, size_t r)
{
	if (r >= bt.num_regs) fail(GFC_ERR_ARG, "register index out of range");
}

void check_test(const gfc_batch &bt, size_t t)
{
	if (t >= bt.count) fail(GFC_ERR_ARG, "test index out of range");
}

void no_capture(const gfc_batch &bt)
{
	if (bt.capturing) fail(GFC_ERR_STATE, "call would synchronise during graph capture");
}

Args make_args(const gfc_batch &bt)
{
	Args a{};
	a.desc = bt.d_desc;
	a.tests = bt.d_tests;
	a.pos = bt.d_pos;
	a.err = bt.d_err;
	a.tab[0] = bt.tab->tab[0];
	a.tab[1] = bt.tab->tab[1];
	if (bt.tabp) a.tab[2] = bt.tabp->tab[2];
	if (bt.twist != nullptr)
	{
		a.twist = 1;
		for (int st = 0; st < 3; ++st)
			for (int pl = 0; pl < 4; ++pl)
			{
				a.tab[st].tf[pl] = bt.twist->tf[st][pl];
				a.tab[st].ti[pl] = bt.twist->ti[st][pl];
			}
	}
	a.n = bt.n;
	a.lr = bt.lr;
	a.num_regs = static_cast<int>(bt.num_regs);
	a.pdl_graph = (bt.packed && (bt.six <= 5)) ? 1 : 0;
	a.ntests = static_cast<uint32_t>(bt.count);
	return a;
}

// Single-CTA kernels: one launch per prime set present (tests sorted by set).
void launch_small(const gfc_batch &bt, const Args &a0, cudaStream_t s, bool prep)
{
	for (int set = 0; set < 2; ++set)
	{
		if (bt.nset[set] == 0) continue;
		Args a = a0;
		a.tests = bt.d_tests + bt.offset[set];
		if (set == 0) small_set<0>(bt.n, a, bt.nset[set], s, prep); else small_set<1>(bt.n, a, bt.nset[set], s, prep);
	}
}

// Cluster-resident squarings: one persistent launch over all tests.
void launch_cluster(gfc_batch &bt, const Args &a, cudaStream_t s)
{
	launch_cluster_n(bt.n, a, static_cast<int>(bt.count), bt.cluster_max, s, false, nullptr);
}

// Raises shared-memory limits of the kernels the current plan uses.
// Whether a six-step plan twists in its middle pass (every row then reads
// the same C - 1 roots): where one direction of the row-pass root tables
// (32 B per point of the packed transform, 24 B per point with a test on
// the three-prime set, else 8 B) reaches 32 MB, and only for the register
// middle passes of 2^3 .. 2^5 rows.  (The tables of every prime are built,
// so a later admission on another prime set stays exact.)  Measured per squaring on one
// B200 (graph replay, twist off -> on): packed n = 21 plan 305 76.0 -> 73.6
// us, n = 22 145.5 -> 138.0, n = 23 plan 305 315.8 -> 298.1; unpacked
// n = 21 plan 105 104.7 -> 99.7; but packed n = 20 plan 303 42.4 -> 44.2
// (its tables stay in L2) and the 64-row pair pass (k_midp, at its
// register limit) 35 -> 47 us per launch at n = 23, more than the rows gain.
bool twist_pays(const gfc_batch &bt)
{
	if ((bt.six < 3) || (bt.six > 5)) return false;
	size_t per_point = 8;
	if (bt.packed) per_point = 32;
	else if (bt.nset[1] > 0) per_point = 24;
	const size_t points = size_t(1) << (bt.packed ? bt.n - 1 : bt.n);
	return per_point * points >= (size_t(32) << 20);
}

void prepare_plan(gfc_batch &bt)
{
	bt.twist = nullptr;
	if (twist_pays(bt))
		bt.twist = bt.packed ? &get_twist(*bt.tabp, true, bt.lr) : &get_twist(*bt.tab, false, bt.lr);
	Args a{};
	a.n = bt.n;
	if (bt.cluster > 0) launch_cluster_n(bt.n, a, 0, 0, nullptr, true, &bt.cluster_max);
	if (bt.packed)
	{
		launch_pcol(bt.six ? MID_LR1 : bt.lr, true, a, 0, nullptr, true);
		if (bt.six) launch_mid(bt.six, false, a, 0, nullptr, true);
		launch_row(bt.n - 1 - bt.lr, a, 0, nullptr, true);
	}
	else if (bt.lr == 0) launch_small(bt, a, nullptr, true);
	else
	{
		launch_col(bt.six ? MID_LR1 : bt.lr, false, a, 0, nullptr, true);
		if (bt.six) launch_mid(bt.six, false, a, 0, nullptr, true);
		launch_row(bt.n - bt.lr, a, 0, nullptr, true);
	}
}

void launch_fixup(gfc_batch &bt, const Args &a, int g)
{
	const unsigned nseg = static_cast<unsigned>(bt.N / SEG);
	const dim3 grid((nseg + FIX_THREADS - 1) / FIX_THREADS, static_cast<unsigned>(g));
	if (bt.packed) launch_pdl(k_pfixup, grid, dim3(FIX_THREADS), 0, bt.stream, a);
	else launch_pdl(k_fixup, grid, dim3(FIX_THREADS), 0, bt.stream, a);
}

// Column passes of the four-step (one kernel) or six-step (2^4-row column
// kernel, then the middle pass; the reverse on the inverse side).
// Packed plans run the same passes on the half-length transform (a.n = n - 1).
Args packed_args(const gfc_batch &bt, const Args &a)
{
	Args p = a;
	p.n = bt.n - 1;
	return p;
}

void launch_cols_fwd(gfc_batch &bt, const Args &a, int g, cudaStream_t s)
{
	if (bt.packed)
	{
		const Args p = packed_args(bt, a);
		launch_pcol(bt.six ? MID_LR1 : bt.lr, false, p, g, s, false);
		if (bt.six) launch_mid(bt.six, false, p, g, s, false, 4);
		return;
	}
	if (bt.six == 0) { launch_col(bt.lr, false, a, g, s, false); return; }
	launch_col(MID_LR1, false, a, g, s, false);
	launch_mid(bt.six, false, a, g, s, false);
}

void launch_cols_inv(gfc_batch &bt, const Args &a, int g, cudaStream_t s)
{
	if (bt.packed)
	{
		const Args p = packed_args(bt, a);
		if (bt.six) launch_mid(bt.six, true, p, g, s, false, 4);
		launch_pcol(bt.six ? MID_LR1 : bt.lr, true, p, g, s, false);
		return;
	}
	if (bt.six == 0) { launch_col(bt.lr, true, a, g, s, false); return; }
	launch_mid(bt.six, true, a, g, s, false);
	launch_col(MID_LR1, true, a, g, s, false);
}

void launch_rows(gfc_batch &bt, const Args &a, int g, cudaStream_t s)
{
	if (bt.packed) launch_row(bt.n - 1 - bt.lr, packed_args(bt, a), g, s, false, 4);
	else launch_row(bt.n - bt.lr, a, g, s, false, 3);
}

// Absorbs the pending segment carries of register bt.pending (k_fixup).
void materialize(gfc_batch &bt)
{
	if (bt.pending < 0) return;
	Args a = make_args(bt);
	a.dup_mode = DUP_NONE;
	a.dst = bt.pending;
	launch_fixup(bt, a, static_cast<int>(bt.count));
	bt.pending = -1;
}

// Four-step squaring / product / forward transform for all tests.  The
// column-forward kernel absorbs pending carries of its source register (and
// writes the fixed digits back); the column-inverse kernel leaves the carries
// of its destination pending.
void fourstep(gfc_batch &bt, Args a)
{
	const int g = static_cast<int>(bt.count);
	a.fix = (bt.pending >= 0 && bt.pending == a.src) ? 1 : 0;
	launch_cols_fwd(bt, a, g, bt.stream);
	if (a.fix) bt.pending = -1;
	launch_rows(bt, a, g, bt.stream);
	if (a.op == OP_FWD) return;
	launch_cols_inv(bt, a, g, bt.stream);
	bt.pending = a.dst;
}

// count squarings of r_0 (dup_mode DUP_NONE / DUP_ALL / DUP_BITS).
void op_square(gfc_batch &bt, int dup_mode, uint32_t count)
{
	if (count == 0) return;
	if (bt.cluster > 0)
	{
		// digits stay in shared memory for all `count` squarings; carries
		// pending on register 0 are absorbed when a test is loaded
		if ((bt.pending >= 0) && (bt.pending != 0)) materialize(bt);
		Args a = make_args(bt);
		a.op = OP_SQUARE; a.dup_mode = dup_mode; a.src = 0; a.dst = 0;
		a.count = static_cast<int>(count);
		a.fix = (bt.pending == 0) ? 1 : 0;
		launch_cluster(bt, a, bt.stream);
		bt.pending = -1;
		return;
	}
	if ((bt.pending >= 0) && ((bt.lr == 0) || (bt.pending != 0))) materialize(bt);
	Args a = make_args(bt);
	a.op = OP_SQUARE; a.dup_mode = dup_mode; a.src = 0; a.dst = 0;
	if (bt.lr == 0)
	{
		a.count = static_cast<int>(count);
		launch_small(bt, a, bt.stream, false);
		return;
	}
	for (uint32_t j = 0; j < count; ++j)
	{
		a.j = (dup_mode == DUP_BITS) ? static_cast<int>(j) : 0;
		fourstep(bt, a);
	}
	if (dup_mode == DUP_BITS)
	{
		const int nt = static_cast<int>(bt.count);
		k_pos_sub<<<(nt + 255) / 256, 256, 0, bt.stream>>>(bt.d_pos, bt.d_tests, nt, static_cast<int>(count));
		after_launch();
	}
}

// r_0 = a r_0^2 for all tests (transform::squareMul, src/transform.h:60).
void op_square_mul(gfc_batch &bt, int32_t m)
{
	if (m == 1 || m == 2) { op_square(bt, (m == 2) ? DUP_ALL : DUP_NONE, 1); return; }
	op_square(bt, DUP_NONE, 1);
	materialize(bt);
	Args a = make_args(bt);
	a.dup_mode = DUP_NONE;
	a.dst = 0;
	const unsigned nseg = static_cast<unsigned>(bt.N / SEG);
	const dim3 grid((nseg + FIX_THREADS - 1) / FIX_THREADS, static_cast<unsigned>(bt.count));
	k_mulscalar<<<grid, FIX_THREADS, 0, bt.stream>>>(a, m);
	after_launch();
	bt.pending = 0;
}

// r_m = transform(r_src) for all tests.
void op_init_multiplicand(gfc_batch &bt, size_t src)
{
	check_reg(bt, src);
	if (bt.lr == 0) materialize(bt);
	Args a = make_args(bt);
	a.op = OP_FWD; a.dup_mode = DUP_NONE; a.src = static_cast<int>(src); a.dst = 0;
	if (bt.lr == 0) launch_small(bt, a, bt.stream, false);
	else fourstep(bt, a);
}

// r_dst = r_0 * r_m for all tests.
void op_mul(gfc_batch &bt, size_t dst)
{
	check_reg(bt, dst);
	if ((bt.pending >= 0) && ((bt.lr == 0) || (bt.pending != 0))) materialize(bt);
	Args a = make_args(bt);
	a.op = OP_MUL; a.dup_mode = DUP_NONE; a.src = 0; a.dst = static_cast<int>(dst);
	if (bt.lr == 0) launch_small(bt, a, bt.stream, false);
	else fourstep(bt, a);
}

// One squaring at a time with events around each kernel (see gfc_batch_time_kernels).
void time_kernels(gfc_batch &bt, uint32_t reps, float *ms)
{
	no_capture(bt);
	if ((bt.pending >= 0) && (bt.pending != 0)) materialize(bt);
	cudaEvent_t ev[5];
	for (auto &e : ev) GFC_CK(cudaEventCreate(&e));
	double acc[5] = { 0, 0, 0, 0, 0 };
	auto span = [&](int i, int j) { float t = 0; GFC_CK(cudaEventElapsedTime(&t, ev[i], ev[j])); return static_cast<double>(t); };
	try
	{
		Args a = make_args(bt);
		a.op = OP_SQUARE; a.dup_mode = DUP_NONE; a.count = 1; a.src = 0; a.dst = 0;
		const int g = static_cast<int>(bt.count);
		for (uint32_t r = 0; r < reps; ++r)
		{
			GFC_CK(cudaEventRecord(ev[0], bt.stream));
			if (bt.cluster > 0)
			{
				a.fix = (bt.pending == 0) ? 1 : 0;
				launch_cluster(bt, a, bt.stream);
				bt.pending = -1;
				GFC_CK(cudaEventRecord(ev[1], bt.stream));
				GFC_CK(cudaEventSynchronize(ev[1]));
				acc[0] += span(0, 1);
			}
			else if (bt.lr == 0)
			{
				launch_small(bt, a, bt.stream, false);
				GFC_CK(cudaEventRecord(ev[1], bt.stream));
				GFC_CK(cudaEventSynchronize(ev[1]));
				acc[0] += span(0, 1);
			}
			else
			{
				a.fix = (bt.pending == 0) ? 1 : 0;
				launch_cols_fwd(bt, a, g, bt.stream);
				GFC_CK(cudaEventRecord(ev[1], bt.stream));
				launch_rows(bt, a, g, bt.stream);
				GFC_CK(cudaEventRecord(ev[2], bt.stream));
				launch_cols_inv(bt, a, g, bt.stream);
				bt.pending = 0;
				GFC_CK(cudaEventRecord(ev[3], bt.stream));
				GFC_CK(cudaEventSynchronize(ev[3]));
				acc[1] += span(0, 1); acc[2] += span(1, 2); acc[3] += span(2, 3);
			}
		}
		if ((bt.lr != 0) && (bt.cluster == 0))
		{
			GFC_CK(cudaEventRecord(ev[3], bt.stream));
			materialize(bt);
			GFC_CK(cudaEventRecord(ev[4], bt.stream));
			GFC_CK(cudaEventSynchronize(ev[4]));
			acc[4] = span(3, 4) * reps;   // one stand-alone fix-up, for reference
		}
	}
	catch (...)
	{
		for (auto &e : ev) cudaEventDestroy(e);
		throw;
	}
	for (auto &e : ev) cudaEventDestroy(e);
	for (int i = 0; i < 5; ++i) ms[i] = static_cast<float>(acc[i] / (reps ? reps : 1));
}

Args all_args(const gfc_batch &bt) { return make_args(bt); }

void op_set(gfc_batch &bt, uint32_t value)
{
	for (size_t i = 0; i < bt.count; ++i)
		if (value > bt.b[i] / 2) fail(GFC_ERR_ARG, "set: value must be <= b/2");
	if (bt.pending == 0) bt.pending = -1;     // register 0 is overwritten
	Args a = all_args(bt);
	a.dst = 0;
	const dim3 grid(static_cast<unsigned>((bt.N + 255) / 256 < 1024 ? (bt.N + 255) / 256 : 1024), static_cast<unsigned>(bt.count));
	k_set<<<grid, 256, 0, bt.stream>>>(a, static_cast<int32_t>(value));
	after_launch();
}

void op_copy(gfc_batch &bt, size_t dst, size_t src)
{
	check_reg(bt, dst); check_reg(bt, src);
	if (dst == src) return;
	if (bt.pending == static_cast<int>(src)) materialize(bt);
	else if (bt.pending == static_cast<int>(dst)) bt.pending = -1;   // overwritten
	Args a = all_args(bt);
	a.dst = static_cast<int>(dst); a.src = static_cast<int>(src);
	const size_t n4 = bt.N / 4;
	const dim3 grid(static_cast<unsigned>((n4 + 255) / 256 < 1024 ? (n4 + 255) / 256 : 1024), static_cast<unsigned>(bt.count));
	k_copy<<<grid, 256, 0, bt.stream>>>(a);
	after_launch();
}

int32_t *reg_ptr(gfc_batch &bt, size_t test, size_t reg) { return bt.regs + (test * bt.num_regs + reg) * bt.N; }

// Waits for the stream and reports (then clears) device-side check failures.
void op_sync(gfc_batch &bt)
{
	no_capture(bt);
	GFC_CK(cudaStreamSynchronize(bt.stream));
	uint32_t err = 0;
	GFC_CK(cudaMemcpy(&err, bt.d_err, sizeof(err), cudaMemcpyDeviceToHost));
	if (err != 0)
	{
		const uint32_t zero = 0;
		GFC_CK(cudaMemcpy(bt.d_err, &zero, sizeof(zero), cudaMemcpyHostToDevice));
		if (err & ERR_GUARD)
			fail(GFC_ERR_STATE, "device check failed: a kernel met a test index or exponent position outside its "
								"batch and skipped the test");
		fail(GFC_ERR_NUMERIC, "device check failed: a segment carry was not absorbed");
	}
}

// |d| <= b/2 + 1 for every digit: d + lim <= 2 lim as one unsigned compare,
// OR-ed without a branch so that the loop vectorises (a scalar loop with an
// early exit took about 4 ms per 4M digits, a tenth of a 64-test block).
void check_digits(const gfc_batch &bt, size_t test, const int32_t *in)
{
	const uint32_t lim = bt.b[test] / 2 + 1, span = 2 * lim;
	uint32_t bad = 0;
	for (size_t i = 0; i < bt.N; ++i) bad |= static_cast<uint32_t>(static_cast<uint32_t>(in[i]) + lim > span);
	if (bad != 0) fail(GFC_ERR_ARG, "digits must satisfy |d| <= b/2 + 1 (balance them first)");
}

gfc_batch *batch_create(const uint32_t *b, size_t count, uint32_t n, size_t num_regs, int device, void *stream)
{
	// the kernels put the test index on grid.y (at most 65535)
	if ((b == nullptr) || (count == 0) || (count > 65535) || (n < 10) || (n > 23) || (num_regs < 1) || (num_regs > 1024))
		fail(GFC_ERR_ARG, "gfc_create: need b, 1 <= count <= 65535, 10 <= n <= 23, 1 <= num_regs <= 1024");
	std::unique_ptr<gfc_batch> bt(new gfc_batch());
	bt->device = device; bt->n = static_cast<int>(n); bt->N = size_t(1) << n; bt->count = count; bt->num_regs = num_regs;
	bt->b.assign(b, b + count);
	bt->set.resize(count);
	for (size_t i = 0; i < count; ++i)
	{
		if ((b[i] < 8) || (b[i] >= (1u << 31))) fail(GFC_ERR_ARG, "base b must satisfy 8 <= b < 2^31");
		const int s = choose_set(b[i], static_cast<int>(n));
		if (s < 0) fail(GFC_ERR_RANGE, "(b, n) is outside the exact range of the RNS prime sets");
		bt->set[i] = s;
		bt->nset[s]++;
	}
	bt->offset[0] = 0; bt->offset[1] = bt->nset[0];
	apply_plan(*bt, default_plan(bt->n));

	GFC_CK(cudaSetDevice(device));
	if (stream != nullptr) bt->stream = static_cast<cudaStream_t>(stream);
	else { GFC_CK(cudaStreamCreateWithFlags(&bt->stream, cudaStreamNonBlocking)); bt->own_stream = true; }
	bt->tab = get_tables(device, bt->n);

	const size_t N = bt->N;
	auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
	const size_t s_regs = al(count * num_regs * N * 4), s_pl = al(count * 3 * N * 4), s_zp = s_pl;
	const size_t s_car = al(count * (N / SEG) * 8 * PK_CARRY), s_desc = al(count * sizeof(TestDesc)), s_tests = al(count * 4);
	const size_t s_pos = al(count * 8), s_err = 256;
	bt->mem_bytes = s_regs + s_pl + s_zp + s_car + s_desc + s_tests + s_pos + s_err;
	bt->mem = dev_alloc(device, bt->mem_bytes, bt->stream);
	char *p = static_cast<char *>(bt->mem);
	bt->regs = reinterpret_cast<int32_t *>(p); p += s_regs;
	bt->planes = reinterpret_cast<uint32_t *>(p); p += s_pl;
	bt->zp = reinterpret_cast<uint32_t *>(p); p += s_zp;
	bt->carry = reinterpret_cast<int64_t *>(p); p += s_car;
	bt->d_desc = reinterpret_cast<TestDesc *>(p); p += s_desc;
	bt->d_tests = reinterpret_cast<int32_t *>(p); p += s_tests;
	bt->d_pos = reinterpret_cast<int64_t *>(p); p += s_pos;
	bt->d_err = reinterpret_cast<uint32_t *>(p);
	GFC_CK(cudaMemsetAsync(bt->mem, 0, bt->mem_bytes, bt->stream));

	bt->h_desc.resize(count);
	bt->ebits.assign(count, nullptr);
	std::vector<int32_t> tests;
	for (int s = 0; s < 2; ++s)
		for (size_t i = 0; i < count; ++i)
			if (bt->set[i] == s) tests.push_back(static_cast<int32_t>(i));
	for (size_t i = 0; i < count; ++i)
	{
		TestDesc &d = bt->h_desc[i];
		d.regs = bt->regs + i * num_regs * N;
		d.planes = bt->planes + i * 3 * N;
		d.zp = bt->zp + i * 3 * N;
		d.carry = bt->carry + i * (N / SEG) * PK_CARRY;
		d.ebits = nullptr;
		d.b = b[i];
		d.set = bt->set[i];
		d.ck = carry_constants(b[i], bt->set[i]);
	}
	GFC_CK(cudaMemcpyAsync(bt->d_desc, bt->h_desc.data(), count * sizeof(TestDesc), cudaMemcpyHostToDevice, bt->stream));
	GFC_CK(cudaMemcpyAsync(bt->d_tests, tests.data(), count * sizeof(int32_t), cudaMemcpyHostToDevice, bt->stream));
	std::vector<int64_t> pos(count, -1);
	GFC_CK(cudaMemcpyAsync(bt->d_pos, pos.data(), count * sizeof(int64_t), cudaMemcpyHostToDevice, bt->stream));
	GFC_CK(cudaStreamSynchronize(bt->stream));
	const size_t pmin = packed_min_tests(bt->n);
	bool packable = (pmin > 0) && (count >= pmin);
	for (size_t i = 0; packable && (i < count); ++i) packable = packed_ok(b[i], bt->n);
	if (packable)
	{
		set_packed(*bt, true);
		apply_plan(*bt, default_packed_plan(bt->n, count));
	}
	else if ((bt->n >= 12) && (bt->n <= SMALL_MAX_LOGN) && (count <= CLUSTER_MAX_TESTS))
		apply_plan(*bt, PLAN_CLUSTER);
	prepare_plan(*bt);
	return bt.release();
}

// ---- autotuner

// Every plan the engine accepts at size n, in the order the tuner tries them:
// single-CTA, cluster, four-step, packed four-step, packed six-step, six-step.
std::vector<int> plan_candidates(int n)
{
	std::vector<int> out;
	auto add = [&](int p) { if (plan_valid(n, p)) out.push_back(p); };
	add(0);
	add(PLAN_CLUSTER);
	for (int lr = 3; lr <= 10; ++lr) add(lr);
	for (int l = 3; l <= 4; ++l) add(PLAN_PACKED + l);
	for (int l2 = 3; l2 <= 7; ++l2) add(PLAN_PACKED_SIX + l2);
	for (int l2 = 3; l2 <= 7; ++l2) add(PLAN_SIX + l2);
	return out;
}

void set_plan_checked(gfc_batch &bt, int lr);

// Device time of one batch squaring under each candidate plan: `squarings`
// squarings of register 0 captured into a CUDA graph, replayed `replays`
// times between CUDA events on the batch stream, minimum taken.  Plans the
// batch cannot take (a base outside the packed range) are skipped.  Sets the
// fastest (ties: the lower code) and clears register 0.  Squares register 0 in
// place: tune a batch before loading its tests.
void op_tune(gfc_batch &bt, uint32_t squarings, uint32_t replays, int32_t *plans, float *us, size_t cap, size_t *count,
			 int32_t *best)
{
	no_capture(bt);
	const std::vector<int> cand = plan_candidates(bt.n);
	cudaEvent_t e0 = nullptr, e1 = nullptr;
	GFC_CK(cudaEventCreate(&e0));
	GFC_CK(cudaEventCreate(&e1));
	std::vector<std::pair<int, float>> got;
	try
	{
		for (int p : cand)
		{
			try { set_plan_checked(bt, p); }
			catch (const Error &e) { if ((e.code == GFC_ERR_ARG) || (e.code == GFC_ERR_RANGE)) continue; throw; }
			materialize(bt);
			cudaGraph_t graph = nullptr;
			cudaGraphExec_t exec = nullptr;
			bt.capturing = true;
			GFC_CK(cudaStreamBeginCapture(bt.stream, cudaStreamCaptureModeThreadLocal));
			const uint64_t l0 = g_launches.load();
			try
			{
				op_square(bt, DUP_NONE, squarings);
				materialize(bt);
			}
			catch (...)
			{
				cudaStreamEndCapture(bt.stream, &graph);
				if (graph != nullptr) cudaGraphDestroy(graph);
				bt.capturing = false;
				throw;
			}
			const uint64_t kernels = g_launches.load() - l0;
			g_launches.fetch_sub(kernels);
			bt.capturing = false;
			GFC_CK(cudaStreamEndCapture(bt.stream, &graph));
			float best_ms = 0;
			try
			{
				GFC_CK(cudaGraphInstantiate(&exec, graph, 0));
				GFC_CK(cudaGraphLaunch(exec, bt.stream));
				g_launches.fetch_add(kernels);
				for (uint32_t r = 0; r < replays; ++r)
				{
					GFC_CK(cudaEventRecord(e0, bt.stream));
					GFC_CK(cudaGraphLaunch(exec, bt.stream));
					g_launches.fetch_add(kernels);
					GFC_CK(cudaEventRecord(e1, bt.stream));
					GFC_CK(cudaEventSynchronize(e1));
					float ms = 0;
					GFC_CK(cudaEventElapsedTime(&ms, e0, e1));
					if ((r == 0) || (ms < best_ms)) best_ms = ms;
				}
			}
			catch (...)
			{
				if (exec != nullptr) cudaGraphExecDestroy(exec);
				cudaGraphDestroy(graph);
				throw;
			}
			cudaGraphExecDestroy(exec);
			cudaGraphDestroy(graph);
			got.emplace_back(p, 1000.0f * best_ms / static_cast<float>(squarings));
		}
	}
	catch (...)
	{
		cudaEventDestroy(e0); cudaEventDestroy(e1);
		throw;
	}
	cudaEventDestroy(e0); cudaEventDestroy(e1);
	if (got.empty()) fail(GFC_ERR_RANGE, "tune: no plan accepts this batch");
	size_t bi = 0;
	for (size_t i = 1; i < got.size(); ++i)
		if ((got[i].second < got[bi].second) || ((got[i].second == got[bi].second) && (got[i].first < got[bi].first))) bi = i;
	set_plan_checked(bt, got[bi].first);
	op_set(bt, 0);
	GFC_CK(cudaStreamSynchronize(bt.stream));
	for (size_t i = 0; (i < got.size()) && (i < cap); ++i)
	{
		if (plans != nullptr) plans[i] = got[i].first;
		if (us != nullptr) us[i] = got[i].second;
	}
	*count = got.size();
	*best = got[bi].first;
}

// ---- reserved slots: staged, asynchronous admission (gfc_batch_reserve)

struct PinSlot
{
	TestDesc *desc;
	int64_t *pos;
	uint32_t *words;
};

PinSlot pin_slot(const gfc_batch &bt, size_t test)
{
	char *p = bt.h_pin + test * bt.pin_slot;
	return { reinterpret_cast<TestDesc *>(p), reinterpret_cast<int64_t *>(p + sizeof(TestDesc)),
			 reinterpret_cast<uint32_t *>(p + sizeof(TestDesc) + sizeof(int64_t)) };
}

int32_t *pin_tests(const gfc_batch &bt) { return reinterpret_cast<int32_t *>(bt.h_pin + bt.count * bt.pin_slot); }
int32_t *pin_one(const gfc_batch &bt) { return pin_tests(bt) + bt.count; }

void op_reserve(gfc_batch &bt, uint64_t max_bits)
{
	if (bt.res_bits != 0) fail(GFC_ERR_STATE, "reserve: the batch is already reserved");
	if ((max_bits == 0) || (max_bits > (uint64_t(1) << 40))) fail(GFC_ERR_ARG, "reserve: need 1 <= max_bits <= 2^40");
	no_capture(bt);
	const size_t words = (((max_bits + 31) / 32) + 3) & ~size_t(3);        // 16-byte multiple per slot
	const size_t slot = (sizeof(TestDesc) + sizeof(int64_t) + 4 * words + 15) & ~size_t(15);
	bt.d_eres = static_cast<uint32_t *>(dev_alloc(bt.device, bt.count * words * sizeof(uint32_t), bt.stream));
	GFC_CK(cudaMemsetAsync(bt.d_eres, 0, bt.count * words * sizeof(uint32_t), bt.stream));
	bt.h_pin = static_cast<char *>(pinned_get(bt.count * slot + (bt.count + 1) * sizeof(int32_t)));
	if (bt.h_pin == nullptr) fail(GFC_ERR_CUDA, "reserve: no page-locked host memory for the staging");
	bt.res_words = words;
	bt.pin_slot = slot;
	*pin_one(bt) = 1;
	bt.slot_ev.assign(bt.count + 1, nullptr);          // one per slot, then one for the tests list
	for (cudaEvent_t &e : bt.slot_ev) GFC_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
	GFC_CK(cudaStreamSynchronize(bt.stream));
	bt.res_bits = max_bits;
}

// Staging of slot `test` is rewritten only after its previous staged copies
// ran (they ran long ago whenever the slot held a test for a block).
void staging_free(gfc_batch &bt, size_t k) { GFC_CK(cudaEventSynchronize(bt.slot_ev[k])); }

// Exponent of a reserved slot: words and position through the slot's pinned
// staging, the descriptor's exponent pointer into the reserved buffer.
void stage_exponent(gfc_batch &bt, size_t test, const uint32_t *words, uint64_t nbits)
{
	staging_free(bt, test);
	const PinSlot ps = pin_slot(bt, test);
	const size_t nw = (nbits + 31) / 32;
	std::memcpy(ps.words, words, nw * sizeof(uint32_t));
	TestDesc &d = bt.h_desc[test];
	d.ebits = bt.d_eres + test * bt.res_words;
	d.ewords = bt.res_words;
	*ps.desc = d;
	*ps.pos = static_cast<int64_t>(nbits) - 1;
	GFC_CK(cudaMemcpyAsync(const_cast<uint32_t *>(d.ebits), ps.words, nw * sizeof(uint32_t), cudaMemcpyHostToDevice, bt.stream));
	GFC_CK(cudaMemcpyAsync(bt.d_desc + test, ps.desc, sizeof(TestDesc), cudaMemcpyHostToDevice, bt.stream));
	GFC_CK(cudaMemcpyAsync(bt.d_pos + test, ps.pos, sizeof(int64_t), cudaMemcpyHostToDevice, bt.stream));
	GFC_CK(cudaEventRecord(bt.slot_ev[test], bt.stream));
}

// A new test in a reserved slot: base, r_0 = r_1 = 1, exponent, position;
// everything enqueued on the batch stream.
void op_admit(gfc_batch &bt, size_t test, uint32_t b, const uint32_t *words, uint64_t nbits)
{
	check_test(bt, test);
	no_capture(bt);
	if (bt.res_bits == 0) fail(GFC_ERR_STATE, "admit: reserve the batch first (gfc_batch_reserve)");
	if ((nbits == 0) || (nbits > bt.res_bits)) fail(GFC_ERR_ARG, "admit: need 1 <= nbits <= the reserved bits");
	if ((b < 8) || (b >= (1u << 31))) fail(GFC_ERR_ARG, "admit: base b must satisfy 8 <= b < 2^31");
	const int s = choose_set(b, bt.n);
	if (s < 0) fail(GFC_ERR_RANGE, "admit: (b, n) is outside the exact range of the RNS prime sets");
	if (bt.packed && !packed_ok(b, bt.n)) fail(GFC_ERR_RANGE, "admit: base outside the range of packed digits");
	materialize(bt);
	if (s != bt.set[test])
	{
		// prime-set order of the per-set launches (single-CTA plan)
		bt.sets_version++;
		bt.nset[bt.set[test]]--;
		bt.set[test] = s;
		bt.nset[s]++;
		bt.offset[0] = 0; bt.offset[1] = bt.nset[0];
		if (bt.lr == 0)
		{
			// the per-set launches read the tests in prime-set order; the
			// staging of the previous order is rewritten after its copy ran
			// (a wait for the block in flight when two admissions of one
			// window change sets)
			staging_free(bt, bt.count);
			int32_t *tl = pin_tests(bt);
			size_t k = 0;
			for (int q = 0; q < 2; ++q)
				for (size_t i = 0; i < bt.count; ++i)
					if (bt.set[i] == q) tl[k++] = static_cast<int32_t>(i);
			GFC_CK(cudaMemcpyAsync(bt.d_tests, tl, bt.count * sizeof(int32_t), cudaMemcpyHostToDevice, bt.stream));
			GFC_CK(cudaEventRecord(bt.slot_ev[bt.count], bt.stream));
			prepare_plan(bt);
		}
		else bt.tests_sorted = false;   // every other launch covers all tests in any order
	}
	bt.b[test] = b;
	TestDesc &d = bt.h_desc[test];
	d.b = b;
	d.set = bt.packed ? 2 : s;
	d.ck = carry_constants(b, bt.packed ? 1 : s);
	if (bt.packed) d.pk = pack_constants(b);
	// registers 0 and 1 (contiguous) = 1, no pending segment carries
	int32_t *r = reg_ptr(bt, test, 0);
	const size_t nr = (bt.num_regs >= 2) ? 2 : 1;
	GFC_CK(cudaMemsetAsync(r, 0, nr * bt.N * sizeof(int32_t), bt.stream));
	for (size_t k = 0; k < nr; ++k)
		GFC_CK(cudaMemcpyAsync(r + k * bt.N, pin_one(bt), sizeof(int32_t), cudaMemcpyHostToDevice, bt.stream));
	GFC_CK(cudaMemsetAsync(d.carry, 0, (bt.N / SEG) * PK_CARRY * sizeof(int64_t), bt.stream));
	stage_exponent(bt, test, words, nbits);
}

void set_plan_checked(gfc_batch &bt, int lr)
{
	if (!plan_valid(bt.n, lr)) fail(GFC_ERR_ARG, "set_plan: invalid plan for this n");
	const bool packed = lr > PLAN_PACKED;   // plans 200 + lr and 300 + lr2
	if (packed)
		for (size_t i = 0; i < bt.count; ++i)
			if (!packed_ok(bt.b[i], bt.n)) fail(GFC_ERR_RANGE, "set_plan: a base is outside the range of packed digits");
	no_capture(bt);
	materialize(bt);                 // pending carries are in the current plan's format
	GFC_CK(cudaStreamSynchronize(bt.stream));
	if (packed != bt.packed) set_packed(bt, packed);
	apply_plan(bt, lr);
	if ((bt.lr == 0) && !bt.tests_sorted)
	{
		std::vector<int32_t> tests;
		for (int q = 0; q < 2; ++q)
			for (size_t i = 0; i < bt.count; ++i)
				if (bt.set[i] == q) tests.push_back(static_cast<int32_t>(i));
		GFC_CK(cudaMemcpy(bt.d_tests, tests.data(), bt.count * sizeof(int32_t), cudaMemcpyHostToDevice));
		bt.tests_sorted = true;
	}
	prepare_plan(bt);
}

template <class F>
int guard(F &&f)
{
	try
	{
		f();
		return GFC_OK;
	}
	catch (const Error &e)
	{
		g_err = e.msg;
		return e.code;
	}
	catch (const std::exception &e)
	{
		g_err = e.what();
		return GFC_ERR_CUDA;
	}
}

#define GFC_NULLCHK(p) \
	if ((p) == nullptr) fail(GFC_ERR_ARG, "null handle or pointer")

}  // namespace

// ------------------------------------------------------------------ C ABI

#define GFC_API extern "C" __attribute__((visibility("default")))

// The message gfc_last_error returns on this thread, for the other sources of
// the library (gf_server_cuda.cpp).
void gfc_internal_set_error(const char *msg) { g_err = (msg != nullptr) ? msg : ""; }

// Page-locked host memory from the library's cache (nullptr when CUDA
// refuses), and its return once no copy uses it.
void *gfc_internal_pinned_get(size_t bytes) { return pinned_get(bytes); }
void gfc_internal_pinned_put(void *p) { pinned_put(p); }

// A server keeps up to `bytes` of freed device memory in each device pool
// and (at most 32 GB of) freed pinned memory for the pools it opens next;
// when the last server ends, the pools and the cache give everything back.
void gfc_internal_retain(bool on, size_t bytes)
{
	MemState &m = mem_state();
	std::vector<void *> drop;
	{
		std::lock_guard<std::mutex> l(m.mu);
		m.retainers += on ? 1 : -1;
		if (m.retainers < 0) m.retainers = 0;
		if (on) m.retain = std::max(m.retain, bytes);
		else if (m.retainers == 0) m.retain = 0;
		uint64_t keep = m.retain;
		for (auto &pd : m.pools)
		{
			cudaMemPoolSetAttribute(pd.second, cudaMemPoolAttrReleaseThreshold, &keep);
			if (keep == 0) cudaMemPoolTrimTo(pd.second, 0);
		}
		while (m.pinned_cached > pinned_cap(m))
		{
			auto it = std::prev(m.pinned_free.end());
			m.pinned_cached -= it->first;
			m.pinned.erase(it->second);
			drop.push_back(it->second);
			m.pinned_free.erase(it);
		}
	}
	for (void *p : drop) cudaFreeHost(p);
}

GFC_API const char *gfc_last_error(void) { return g_err.c_str(); }
GFC_API int gfc_version(void) { return 100; }
GFC_API uint64_t gfc_launch_count(void) { return g_launches.load(); }

// ---- single test

GFC_API int gfc_create(uint32_t b, uint32_t n, size_t num_regs, int device, void *stream, gfc_transform **out)
{
	return guard([&] {
		GFC_NULLCHK(out);
		*out = nullptr;
		*out = batch_create(&b, 1, n, num_regs, device, stream);
	});
}

GFC_API void gfc_destroy(gfc_transform *t) { delete t; }

GFC_API int gfc_set(gfc_transform *t, uint32_t a)
{
	return guard([&] { GFC_NULLCHK(t); cudaSetDevice(t->device); op_set(*t, a); });
}

GFC_API int gfc_square_dup(gfc_transform *t, int dup)
{
	return guard([&] { GFC_NULLCHK(t); cudaSetDevice(t->device); op_square(*t, dup ? DUP_ALL : DUP_NONE, 1); });
}

GFC_API int gfc_square_mul(gfc_transform *t, int32_t a)
{
	return guard([&] { GFC_NULLCHK(t); cudaSetDevice(t->device); op_square_mul(*t, a); });
}

GFC_API int gfc_init_multiplicand(gfc_transform *t, size_t src)
{
	return guard([&] { GFC_NULLCHK(t); cudaSetDevice(t->device); op_init_multiplicand(*t, src); });
}

GFC_API int gfc_mul(gfc_transform *t)
{
	return guard([&] { GFC_NULLCHK(t); cudaSetDevice(t->device); op_mul(*t, 0); });
}

GFC_API int gfc_copy(gfc_transform *t, size_t dst, size_t src)
{
	return guard([&] { GFC_NULLCHK(t); cudaSetDevice(t->device); op_copy(*t, dst, src); });
}

GFC_API int gfc_get_zi(gfc_transform *t, int32_t *zi)
{
	return gfc_batch_get_zi(t, 0, 0, zi);
}

GFC_API int gfc_set_zi(gfc_transform *t, const int32_t *zi)
{
	return gfc_batch_set_zi(t, 0, 0, zi);
}

GFC_API size_t gfc_get_mem_size(const gfc_transform *t) { return (t == nullptr) ? 0 : t->mem_bytes; }

GFC_API size_t gfc_get_cache_size(const gfc_transform *t)
{
	if (t == nullptr) return 0;
	return (t->set[0] == 0 ? 2 : 3) * t->N * sizeof(uint32_t) + t->N * sizeof(int32_t);
}

GFC_API size_t gfc_context_size(const gfc_transform *t, size_t num_regs)
{
	return (t == nullptr) ? 0 : sizeof(uint32_t) + num_regs * t->N * sizeof(int32_t);
}

GFC_API int gfc_save_context(gfc_transform *t, void *buf, size_t size, size_t num_regs)
{
	return guard([&] {
		GFC_NULLCHK(t); GFC_NULLCHK(buf);
		if ((num_regs == 0) || (num_regs > t->num_regs) || (size < gfc_context_size(t, num_regs)))
			fail(GFC_ERR_ARG, "save_context: bad register count or buffer size");
		no_capture(*t);
		cudaSetDevice(t->device);
		const uint32_t kind = GFC_CONTEXT_KIND;
		std::memcpy(buf, &kind, sizeof(kind));
		materialize(*t);
		GFC_CK(cudaMemcpyAsync(static_cast<char *>(buf) + sizeof(kind), t->regs, num_regs * t->N * sizeof(int32_t),
							   cudaMemcpyDeviceToHost, t->stream));
		op_sync(*t);
	});
}

GFC_API int gfc_read_context(gfc_transform *t, const void *buf, size_t size, size_t num_regs)
{
	return guard([&] {
		GFC_NULLCHK(t); GFC_NULLCHK(buf);
		if ((num_regs == 0) || (num_regs > t->num_regs)) fail(GFC_ERR_ARG, "read_context: bad register count");
		uint32_t kind = 0;
		if (size >= sizeof(kind)) std::memcpy(&kind, buf, sizeof(kind));
		if ((kind != GFC_CONTEXT_KIND) || (size != gfc_context_size(t, num_regs)))
			fail(GFC_ERR_STATE, "read_context: context kind or size mismatch");
		const int32_t *d = reinterpret_cast<const int32_t *>(static_cast<const char *>(buf) + sizeof(kind));
		for (size_t r = 0; r < num_regs; ++r) check_digits(*t, 0, d + r * t->N);
		no_capture(*t);
		cudaSetDevice(t->device);
		materialize(*t);
		GFC_CK(cudaMemcpyAsync(t->regs, d, num_regs * t->N * sizeof(int32_t), cudaMemcpyHostToDevice, t->stream));
		op_sync(*t);
	});
}

GFC_API int gfc_width(const gfc_transform *t)
{
	if (t == nullptr) return GFC_ERR_ARG;
	return t->packed ? 4 : (t->set[0] == 0 ? 2 : 3);
}

GFC_API int gfc_sync(gfc_transform *t)
{
	return guard([&] { GFC_NULLCHK(t); cudaSetDevice(t->device); op_sync(*t); });
}

// ---- batches

GFC_API int gfc_batch_create(const uint32_t *b, size_t count, uint32_t n, size_t num_regs, int device, void *stream,
							 gfc_batch **out)
{
	return guard([&] {
		GFC_NULLCHK(out);
		*out = nullptr;
		*out = batch_create(b, count, n, num_regs, device, stream);
	});
}

GFC_API void gfc_batch_destroy(gfc_batch *bt) { delete bt; }
GFC_API size_t gfc_batch_count(const gfc_batch *bt) { return (bt == nullptr) ? 0 : bt->count; }

GFC_API int gfc_batch_set(gfc_batch *bt, uint32_t a)
{
	return guard([&] { GFC_NULLCHK(bt); cudaSetDevice(bt->device); op_set(*bt, a); });
}

GFC_API int gfc_batch_copy(gfc_batch *bt, size_t dst, size_t src)
{
	return guard([&] { GFC_NULLCHK(bt); cudaSetDevice(bt->device); op_copy(*bt, dst, src); });
}

GFC_API int gfc_batch_square(gfc_batch *bt, int dup, uint32_t count)
{
	return guard([&] { GFC_NULLCHK(bt); cudaSetDevice(bt->device); op_square(*bt, dup ? DUP_ALL : DUP_NONE, count); });
}

GFC_API int gfc_batch_set_exponent(gfc_batch *bt, size_t test, const uint32_t *words, uint64_t nbits)
{
	return guard([&] {
		GFC_NULLCHK(bt); GFC_NULLCHK(words);
		check_test(*bt, test);
		no_capture(*bt);
		if (nbits == 0) fail(GFC_ERR_ARG, "set_exponent: empty exponent");
		cudaSetDevice(bt->device);
		if ((bt->res_bits != 0) && (nbits <= bt->res_bits))
		{
			stage_exponent(*bt, test, words, nbits);
			return;
		}
		GFC_CK(cudaStreamSynchronize(bt->stream));
		const size_t nw = (nbits + 31) / 32;
		dev_free(bt->device, bt->ebits[test]);
		bt->ebits[test] = nullptr;
		bt->ebits[test] = static_cast<uint32_t *>(dev_alloc(bt->device, nw * sizeof(uint32_t), bt->stream));
		bt->h_desc[test].ebits = bt->ebits[test];
		bt->h_desc[test].ewords = nw;
		const int64_t pos = static_cast<int64_t>(nbits) - 1;
		GFC_CK(cudaMemcpyAsync(bt->ebits[test], words, nw * sizeof(uint32_t), cudaMemcpyHostToDevice, bt->stream));
		GFC_CK(cudaMemcpyAsync(bt->d_desc + test, &bt->h_desc[test], sizeof(TestDesc), cudaMemcpyHostToDevice, bt->stream));
		GFC_CK(cudaMemcpyAsync(bt->d_pos + test, &pos, sizeof(pos), cudaMemcpyHostToDevice, bt->stream));
		GFC_CK(cudaStreamSynchronize(bt->stream));
	});
}

GFC_API int gfc_batch_reserve(gfc_batch *bt, uint64_t max_bits)
{
	return guard([&] { GFC_NULLCHK(bt); cudaSetDevice(bt->device); op_reserve(*bt, max_bits); });
}

GFC_API int gfc_batch_admit(gfc_batch *bt, size_t test, uint32_t b, const uint32_t *words, uint64_t nbits)
{
	return guard([&] {
		GFC_NULLCHK(bt); GFC_NULLCHK(words);
		cudaSetDevice(bt->device);
		op_admit(*bt, test, b, words, nbits);
	});
}

GFC_API int gfc_batch_get_async(gfc_batch *bt, size_t test, size_t reg, int32_t *out)
{
	return guard([&] {
		GFC_NULLCHK(bt); GFC_NULLCHK(out);
		check_test(*bt, test); check_reg(*bt, reg);
		no_capture(*bt);
		cudaSetDevice(bt->device);
		materialize(*bt);
		GFC_CK(cudaMemcpyAsync(out, reg_ptr(*bt, test, reg), bt->N * sizeof(int32_t), cudaMemcpyDeviceToHost, bt->stream));
	});
}

GFC_API int gfc_batch_set_async(gfc_batch *bt, size_t test, size_t reg, const int32_t *in)
{
	return guard([&] {
		GFC_NULLCHK(bt); GFC_NULLCHK(in);
		check_test(*bt, test); check_reg(*bt, reg);
		check_digits(*bt, test, in);
		no_capture(*bt);
		cudaSetDevice(bt->device);
		materialize(*bt);
		GFC_CK(cudaMemcpyAsync(reg_ptr(*bt, test, reg), in, bt->N * sizeof(int32_t), cudaMemcpyHostToDevice, bt->stream));
	});
}

GFC_API int gfc_width_for(uint32_t b, uint32_t n)
{
	if ((b < 8) || (b >= (1u << 31)) || (n < 8) || (n > 23)) return GFC_ERR_ARG;
	const int s = choose_set(b, static_cast<int>(n));
	return (s < 0) ? GFC_ERR_RANGE : ((s == 0) ? 2 : 3);
}

GFC_API int gfc_packed_range(uint32_t b, uint32_t n)
{
	if ((n < 9) || (n > 23)) return 0;
	return packed_ok(b, static_cast<int>(n)) ? 1 : 0;
}

GFC_API int gfc_plan_candidates(uint32_t n, int32_t *plans, size_t cap, size_t *count)
{
	return guard([&] {
		GFC_NULLCHK(count);
		const std::vector<int> c = plan_candidates(static_cast<int>(n));
		if ((plans == nullptr) && (cap != 0)) fail(GFC_ERR_ARG, "plan_candidates: null output");
		for (size_t i = 0; (i < c.size()) && (i < cap); ++i) plans[i] = c[i];
		*count = c.size();
	});
}

GFC_API int gfc_batch_tune(gfc_batch *bt, uint32_t squarings, uint32_t replays, int32_t *plans, float *us, size_t cap,
						   size_t *count, int32_t *best)
{
	return guard([&] {
		GFC_NULLCHK(bt); GFC_NULLCHK(count); GFC_NULLCHK(best);
		if ((squarings == 0) || (replays == 0)) fail(GFC_ERR_ARG, "tune: need squarings >= 1 and replays >= 1");
		cudaSetDevice(bt->device);
		op_tune(*bt, squarings, replays, plans, us, cap, count, best);
	});
}

GFC_API int gfc_batch_assign(gfc_batch *bt, size_t test, uint32_t b)
{
	return guard([&] {
		GFC_NULLCHK(bt);
		check_test(*bt, test);
		no_capture(*bt);
		if ((b < 8) || (b >= (1u << 31))) fail(GFC_ERR_ARG, "assign: base b must satisfy 8 <= b < 2^31");
		const int s = choose_set(b, bt->n);
		if (s < 0) fail(GFC_ERR_RANGE, "assign: (b, n) is outside the exact range of the RNS prime sets");
		cudaSetDevice(bt->device);
		materialize(*bt);
		GFC_CK(cudaStreamSynchronize(bt->stream));
		if (s != bt->set[test]) bt->sets_version++;
		bt->nset[bt->set[test]]--;
		bt->b[test] = b;
		bt->set[test] = s;
		bt->nset[s]++;
		bt->offset[0] = 0; bt->offset[1] = bt->nset[0];
		std::vector<int32_t> tests;
		for (int k = 0; k < 2; ++k)
			for (size_t i = 0; i < bt->count; ++i)
				if (bt->set[i] == k) tests.push_back(static_cast<int32_t>(i));
		if (bt->packed && !packed_ok(b, bt->n)) fail(GFC_ERR_RANGE, "assign: base outside the range of packed digits");
		TestDesc &d = bt->h_desc[test];
		d.b = b;
		d.set = s;
		d.ck = carry_constants(b, s);
		if (bt->packed)
		{
			d.set = 2;
			d.ck = carry_constants(b, 1);
			d.pk = pack_constants(b);
		}
		GFC_CK(cudaMemcpy(bt->d_desc + test, &d, sizeof(TestDesc), cudaMemcpyHostToDevice));
		GFC_CK(cudaMemcpy(bt->d_tests, tests.data(), bt->count * sizeof(int32_t), cudaMemcpyHostToDevice));
		bt->tests_sorted = true;
		prepare_plan(*bt);
	});
}

GFC_API int gfc_batch_set_pos(gfc_batch *bt, const int64_t *pos)
{
	return guard([&] {
		GFC_NULLCHK(bt); GFC_NULLCHK(pos);
		no_capture(*bt);
		cudaSetDevice(bt->device);
		for (size_t i = 0; i < bt->count; ++i)
			if ((pos[i] >= 0) && (bt->h_desc[i].ebits == nullptr)) fail(GFC_ERR_STATE, "set_pos: test has no exponent");
		GFC_CK(cudaMemcpyAsync(bt->d_pos, pos, bt->count * sizeof(int64_t), cudaMemcpyHostToDevice, bt->stream));
		GFC_CK(cudaStreamSynchronize(bt->stream));
	});
}

GFC_API int gfc_batch_get_pos(gfc_batch *bt, int64_t *pos)
{
	return guard([&] {
		GFC_NULLCHK(bt); GFC_NULLCHK(pos);
		no_capture(*bt);
		cudaSetDevice(bt->device);
		GFC_CK(cudaMemcpyAsync(pos, bt->d_pos, bt->count * sizeof(int64_t), cudaMemcpyDeviceToHost, bt->stream));
		GFC_CK(cudaStreamSynchronize(bt->stream));
	});
}

GFC_API int gfc_batch_square_exp(gfc_batch *bt, uint32_t count)
{
	return guard([&] {
		GFC_NULLCHK(bt);
		cudaSetDevice(bt->device);
		op_square(*bt, DUP_BITS, count);
	});
}

GFC_API int gfc_batch_init_multiplicand(gfc_batch *bt, size_t src)
{
	return guard([&] { GFC_NULLCHK(bt); cudaSetDevice(bt->device); op_init_multiplicand(*bt, src); });
}

GFC_API int gfc_batch_mul(gfc_batch *bt, size_t dst)
{
	return guard([&] { GFC_NULLCHK(bt); cudaSetDevice(bt->device); op_mul(*bt, dst); });
}

GFC_API int gfc_batch_gl_step(gfc_batch *bt)
{
	return guard([&] {
		GFC_NULLCHK(bt);
		if (bt->num_regs < 2) fail(GFC_ERR_STATE, "gl_step needs 2 registers");
		cudaSetDevice(bt->device);
		op_init_multiplicand(*bt, 1);
		op_mul(*bt, 1);
	});
}

GFC_API int gfc_batch_get_zi(gfc_batch *bt, size_t test, size_t reg, int32_t *out)
{
	return guard([&] {
		GFC_NULLCHK(bt); GFC_NULLCHK(out);
		check_test(*bt, test); check_reg(*bt, reg);
		no_capture(*bt);
		cudaSetDevice(bt->device);
		materialize(*bt);
		GFC_CK(cudaMemcpyAsync(out, reg_ptr(*bt, test, reg), bt->N * sizeof(int32_t), cudaMemcpyDeviceToHost, bt->stream));
		op_sync(*bt);
	});
}

GFC_API int gfc_batch_set_zi(gfc_batch *bt, size_t test, size_t reg, const int32_t *in)
{
	return guard([&] {
		GFC_NULLCHK(bt); GFC_NULLCHK(in);
		check_test(*bt, test); check_reg(*bt, reg);
		check_digits(*bt, test, in);
		no_capture(*bt);
		cudaSetDevice(bt->device);
		materialize(*bt);
		GFC_CK(cudaMemcpyAsync(reg_ptr(*bt, test, reg), in, bt->N * sizeof(int32_t), cudaMemcpyHostToDevice, bt->stream));
		GFC_CK(cudaStreamSynchronize(bt->stream));
	});
}

GFC_API int gfc_batch_get_all(gfc_batch *bt, size_t reg, int32_t *out)
{
	return guard([&] {
		GFC_NULLCHK(bt); GFC_NULLCHK(out);
		check_reg(*bt, reg);
		no_capture(*bt);
		cudaSetDevice(bt->device);
		materialize(*bt);
		// registers of one test are contiguous: reg r of test i at (i * num_regs + r) * N
		GFC_CK(cudaMemcpy2DAsync(out, bt->N * sizeof(int32_t), reg_ptr(*bt, 0, reg), bt->num_regs * bt->N * sizeof(int32_t),
								 bt->N * sizeof(int32_t), bt->count, cudaMemcpyDeviceToHost, bt->stream));
		op_sync(*bt);
	});
}

// The digits of every test go to its planes (transform scratch, dead between
// operations), are checked there on the device and copied into the register
// only if every digit of every test is in range: the same refusal as a host
// check, without a pass over the host buffer (two 4M-digit registers per
// 64-test n = 16 block took milliseconds on the host).
GFC_API int gfc_batch_set_all(gfc_batch *bt, size_t reg, const int32_t *in)
{
	return guard([&] {
		GFC_NULLCHK(bt); GFC_NULLCHK(in);
		check_reg(*bt, reg);
		no_capture(*bt);
		cudaSetDevice(bt->device);
		materialize(*bt);
		const size_t N = bt->N;
		uint32_t *bad = bt->d_err + 1;
		GFC_CK(cudaMemsetAsync(bad, 0, sizeof(uint32_t), bt->stream));
		GFC_CK(cudaMemcpy2DAsync(bt->planes, 3 * N * sizeof(int32_t), in, N * sizeof(int32_t), N * sizeof(int32_t),
								 bt->count, cudaMemcpyHostToDevice, bt->stream));
		const dim3 grid(static_cast<unsigned>(std::min<size_t>(N / 1024, 64)), static_cast<unsigned>(bt->count));
		k_check_digits<<<grid, 256, 0, bt->stream>>>(bt->d_desc, bt->n, bad);
		after_launch();
		k_commit_digits<<<grid, 256, 0, bt->stream>>>(bt->d_desc, bt->n, static_cast<int>(reg), bad);
		after_launch();
		uint32_t flag = 0;
		GFC_CK(cudaStreamSynchronize(bt->stream));
		GFC_CK(cudaMemcpy(&flag, bad, sizeof(flag), cudaMemcpyDeviceToHost));
		if (flag != 0) fail(GFC_ERR_ARG, "digits must satisfy |d| <= b/2 + 1 (balance them first)");
	});
}

GFC_API int gfc_batch_set_plan(gfc_batch *bt, int lr)
{
	return guard([&] {
		GFC_NULLCHK(bt);
		cudaSetDevice(bt->device);
		set_plan_checked(*bt, lr);
	});
}

GFC_API int gfc_batch_plan(const gfc_batch *bt)
{
	if (bt == nullptr) return GFC_ERR_ARG;
	if (bt->packed) return (bt->six > 0) ? PLAN_PACKED_SIX + bt->six : PLAN_PACKED + bt->lr;
	if (bt->cluster > 0) return PLAN_CLUSTER;
	return (bt->six > 0) ? PLAN_SIX + bt->six : bt->lr;
}

GFC_API int gfc_batch_widths(const gfc_batch *bt, int32_t *w)
{
	return guard([&] {
		GFC_NULLCHK(bt); GFC_NULLCHK(w);
		for (size_t i = 0; i < bt->count; ++i) w[i] = bt->packed ? 4 : ((bt->set[i] == 0) ? 2 : 3);
	});
}

GFC_API int gfc_batch_time_kernels(gfc_batch *bt, uint32_t reps, float *ms)
{
	return guard([&] { GFC_NULLCHK(bt); GFC_NULLCHK(ms); cudaSetDevice(bt->device); time_kernels(*bt, reps, ms); });
}

GFC_API int gfc_batch_sync(gfc_batch *bt)
{
	return guard([&] { GFC_NULLCHK(bt); cudaSetDevice(bt->device); op_sync(*bt); });
}

GFC_API void *gfc_batch_stream(gfc_batch *bt) { return (bt == nullptr) ? nullptr : static_cast<void *>(bt->stream); }

GFC_API int gfc_batch_capture_begin(gfc_batch *bt)
{
	return guard([&] {
		GFC_NULLCHK(bt);
		no_capture(*bt);
		cudaSetDevice(bt->device);
		materialize(*bt);   // a graph starts and ends with every register materialised
		GFC_CK(cudaStreamBeginCapture(bt->stream, cudaStreamCaptureModeThreadLocal));
		bt->capturing = true;
		bt->capture_start = g_launches.load();
	});
}

GFC_API int gfc_batch_capture_end(gfc_batch *bt, gfc_graph **out)
{
	return guard([&] {
		GFC_NULLCHK(bt); GFC_NULLCHK(out);
		*out = nullptr;
		if (!bt->capturing) fail(GFC_ERR_STATE, "capture_end without capture_begin");
		cudaSetDevice(bt->device);
		try { materialize(*bt); } catch (...) { }
		bt->capturing = false;
		std::unique_ptr<gfc_graph> g(new gfc_graph());
		g->batch = bt; g->device = bt->device; g->stream = bt->stream;
		g->sets_version = bt->sets_version; g->per_set = (bt->lr == 0);
		// recorded launches are counted when the graph runs, not here
		g->kernels = g_launches.load() - bt->capture_start;
		g_launches.fetch_sub(g->kernels);
		GFC_CK(cudaStreamEndCapture(bt->stream, &g->graph));
		GFC_CK(cudaGraphInstantiate(&g->exec, g->graph, 0));
		*out = g.release();
	});
}

GFC_API int gfc_graph_launch(gfc_graph *g)
{
	return guard([&] {
		GFC_NULLCHK(g);
		cudaSetDevice(g->device);
		if ((g->batch != nullptr) && g->per_set && (g->batch->sets_version != g->sets_version))
			fail(GFC_ERR_STATE, "graph_launch: a test changed prime set since capture; capture again");
		if (g->batch != nullptr) materialize(*g->batch);
		GFC_CK(cudaGraphLaunch(g->exec, g->stream));
		g_launches.fetch_add(g->kernels);
	});
}

GFC_API void gfc_graph_destroy(gfc_graph *g) { delete g; }

// ------------------------------------------------------------------ squaring without allocation
//
// gfc_square_noalloc runs the four-step squaring with all of its scratch
// (root tables, transform planes, segment carries, test descriptor) in one
// file-scope device array instead of memory from cudaMalloc.  It exists for
// callers that cannot allocate device memory when they square: code running
// inside another runtime's memory pool or allocator lock, processes whose
// device-memory budget is fixed at start-up, and hosts that forbid
// allocation after initialisation.  The array is part of the library image,
// so every GPU that loads the library holds it until the process exits.

namespace {

constexpr int NA_MIN_LOGN = 12, NA_MAX_LOGN = 16, NA_LR = 4;
constexpr size_t NA_N = size_t(1) << NA_MAX_LOGN;
// Layout in 32-bit words.
constexpr size_t NA_OFF_TAB = 0;                                  // 5 primes x (forward, inverse) x N entries
constexpr size_t NA_TAB_WORDS = 2 * (2 * 1 + 3 * 2) * NA_N;       // 1 word per entry (32-bit primes), 2 (31-bit)
constexpr size_t NA_OFF_PLANES = NA_OFF_TAB + NA_TAB_WORDS;       // 3 planes x N
constexpr size_t NA_OFF_CARRY = NA_OFF_PLANES + 3 * NA_N;         // N/16 int64 carries
constexpr size_t NA_OFF_DESC = NA_OFF_CARRY + NA_N / 8;           // one TestDesc
constexpr size_t NA_OFF_MISC = NA_OFF_DESC + 128;                 // test index, position, error word
constexpr size_t NA_WORDS = NA_OFF_MISC + 64;                     // 5.01 MB
static_assert(sizeof(TestDesc) <= 128 * sizeof(uint32_t), "descriptor slot");

static __device__ __align__(256) uint32_t g_na_scratch[NA_WORDS];

constexpr int NA_MAX_DEVICES = 64;
struct NaDevice
{
	uint32_t *base = nullptr;   // device address of g_na_scratch on this device
	int tab_n = 0;              // n of the root tables currently stored
};
std::mutex g_na_mu;
NaDevice g_na_dev[NA_MAX_DEVICES];
uint32_t g_na_pw[NA_N + 1], g_na_fw[2 * NA_N], g_na_iv[2 * NA_N];   // host staging for the root tables

// Word offset of prime s's forward table in the scratch array (its inverse
// table follows it).
size_t na_tab_off(int s)
{
	size_t o = NA_OFF_TAB;
	for (int i = 0; i < s; ++i) o += 2 * root_words(kPrime[i]) * NA_N;
	return o;
}

// Smallest generator of (Z/pZ)* without heap use (p - 1 has < 10 prime factors).
uint32_t na_primitive_root(uint32_t p)
{
	uint32_t f[16];
	int nf = 0;
	uint32_t m = p - 1;
	for (uint32_t q = 2; static_cast<uint64_t>(q) * q <= m; ++q)
		if (m % q == 0) { f[nf++] = q; while (m % q == 0) m /= q; }
	if (m > 1) f[nf++] = m;
	for (uint32_t g = 2;; ++g)
	{
		bool ok = true;
		for (int i = 0; i < nf; ++i) if (powmod_h(g, (p - 1) / f[i], p) == 1) { ok = false; break; }
		if (ok) return g;
	}
}

// The root tables of build_roots_device(), built on the host into the staging arrays.
void na_build_roots(uint32_t p, int n)
{
	const uint32_t N = 1u << n;
	const uint32_t psi = powmod_h(na_primitive_root(p), (p - 1) / (2ull * N), p);
	g_na_pw[0] = 1;
	for (uint32_t i = 1; i <= N; ++i) g_na_pw[i] = mulmod_h(g_na_pw[i - 1], psi, p);
	for (uint32_t k = 1; k < N; ++k)
	{
		const uint32_t e = bitrev(k, n);
		put_root(g_na_fw, k, g_na_pw[e], p);
		put_root(g_na_iv, k, p - g_na_pw[N - e], p);
	}
	const uint32_t R1 = static_cast<uint32_t>((uint64_t(1) << 32) % p);
	const uint32_t c = mulmod_h(mulmod_h(R1, R1, p), powmod_h(N % p, p - 2, p), p);
	g_na_fw[0] = c;
	g_na_iv[0] = mulmod_h(p - g_na_pw[N / 2], c, p);
	if (root_words(p) == 2) { g_na_fw[1] = 0; g_na_iv[1] = 0; }
}

// Per-device set-up (first call on a device): the device address of the
// scratch array, and the root tables for n whenever n changes.
NaDevice &na_setup(int device, int n)
{
	if ((device < 0) || (device >= NA_MAX_DEVICES)) fail(GFC_ERR_ARG, "square_noalloc: device ordinal out of range");
	NaDevice &nd = g_na_dev[device];
	if (nd.base == nullptr)
	{
		void *p = nullptr;
		const cudaError_t e = cudaGetSymbolAddress(&p, g_na_scratch);
		if (e != cudaSuccess) fail(GFC_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
		nd.base = static_cast<uint32_t *>(p);
	}
	if (nd.tab_n != n)
	{
		const size_t N = size_t(1) << n;
		nd.tab_n = 0;
		for (int s = 0; s < 5; ++s)
		{
			na_build_roots(kPrime[s], n);
			const size_t rw = root_words(kPrime[s]);
			GFC_CK(cudaMemcpy(nd.base + na_tab_off(s), g_na_fw, rw * N * sizeof(uint32_t), cudaMemcpyHostToDevice));
			GFC_CK(cudaMemcpy(nd.base + na_tab_off(s) + rw * NA_N, g_na_iv, rw * N * sizeof(uint32_t),
							  cudaMemcpyHostToDevice));
		}
		nd.tab_n = n;
	}
	return nd;
}

}  // namespace

GFC_API int gfc_square_noalloc(const int32_t *in, int32_t *out, uint32_t b, uint32_t n, int dup, uint32_t count,
							   int device, void *stream)
{
	return guard([&] {
		if ((in == nullptr) || (out == nullptr)) fail(GFC_ERR_ARG, "square_noalloc: null digit pointer");
		if ((n < NA_MIN_LOGN) || (n > NA_MAX_LOGN))
			fail(GFC_ERR_ARG, "square_noalloc: n must satisfy 12 <= n <= 16 (size of the static scratch array)");
		{
			// the device-to-device copy below needs in == out or disjoint ranges
			const uintptr_t pi = reinterpret_cast<uintptr_t>(in), po = reinterpret_cast<uintptr_t>(out);
			const uintptr_t bytes = (uintptr_t(1) << n) * sizeof(int32_t);
			if ((pi != po) && (((pi < po) ? po - pi : pi - po) < bytes))
				fail(GFC_ERR_ARG, "square_noalloc: in and out must be equal or disjoint");
		}
		if ((b < 8) || (b >= (1u << 31))) fail(GFC_ERR_ARG, "square_noalloc: base b must satisfy 8 <= b < 2^31");
		const int set = choose_set(b, static_cast<int>(n));
		if (set < 0) fail(GFC_ERR_RANGE, "square_noalloc: (b, n) is outside the exact range of the RNS prime sets");
		std::lock_guard<std::mutex> lock(g_na_mu);
		GFC_CK(cudaSetDevice(device));
		NaDevice &nd = na_setup(device, static_cast<int>(n));
		const cudaStream_t s = static_cast<cudaStream_t>(stream);
		const size_t N = size_t(1) << n;
		uint32_t *const base = nd.base;

		// descriptor of the single test, read by the kernels from the scratch array
		TestDesc d{};
		d.regs = out;
		d.planes = base + NA_OFF_PLANES;
		d.zp = base + NA_OFF_PLANES;
		d.carry = reinterpret_cast<int64_t *>(base + NA_OFF_CARRY);
		d.ebits = nullptr;
		d.ck = carry_constants(b, set);
		d.b = b;
		d.set = set;
		struct { int32_t test; int32_t pad; int64_t pos; uint32_t err; } misc = { 0, 0, 0, 0 };
		GFC_CK(cudaMemcpyAsync(base + NA_OFF_DESC, &d, sizeof(d), cudaMemcpyHostToDevice, s));
		// the error word must start at zero; planes and carries are written before they are read
		GFC_CK(cudaMemcpyAsync(base + NA_OFF_MISC, &misc, sizeof(misc), cudaMemcpyHostToDevice, s));
		if (in != out) GFC_CK(cudaMemcpyAsync(out, in, N * sizeof(int32_t), cudaMemcpyDeviceToDevice, s));

		Args a{};
		a.desc = reinterpret_cast<const TestDesc *>(base + NA_OFF_DESC);
		a.tests = reinterpret_cast<const int32_t *>(base + NA_OFF_MISC);
		a.pos = reinterpret_cast<int64_t *>(base + NA_OFF_MISC + 2);
		a.err = base + NA_OFF_MISC + 4;
		const int slot0[2] = { 0, 2 };
		for (int st = 0; st < 2; ++st)
			for (int pl = 0; pl < 3; ++pl)
			{
				const int k = (st == 0 && pl == 2) ? 1 : slot0[st] + pl;
				a.tab[st].fw[pl] = base + na_tab_off(k);
				a.tab[st].iv[pl] = base + na_tab_off(k) + root_words(kPrime[k]) * NA_N;
			}
		a.n = static_cast<int>(n);
		a.lr = NA_LR;
		a.num_regs = 1;
		a.op = OP_SQUARE;
		a.dup_mode = dup ? DUP_ALL : DUP_NONE;

		const int lc = static_cast<int>(n) - NA_LR;
		launch_col(NA_LR, false, a, 0, nullptr, true);
		launch_row(lc, a, 0, nullptr, true);
		for (uint32_t j = 0; j < count; ++j)
		{
			a.fix = (j > 0) ? 1 : 0;   // carries of the previous squaring are absorbed on load
			launch_col(NA_LR, false, a, 1, s, false);
			launch_row(lc, a, 1, s, false);
			launch_col(NA_LR, true, a, 1, s, false);
		}
		if (count > 0)
		{
			const dim3 grid(static_cast<unsigned>((N / SEG + 255) / 256), 1u);
			k_fixup<<<grid, 256, 0, s>>>(a);
			after_launch();
		}
		uint32_t err = 0;
		GFC_CK(cudaMemcpyAsync(&err, base + NA_OFF_MISC + 4, sizeof(err), cudaMemcpyDeviceToHost, s));
		GFC_CK(cudaStreamSynchronize(s));
		if (err != 0) fail(GFC_ERR_NUMERIC, "square_noalloc: a segment carry was not absorbed");
	});
}
