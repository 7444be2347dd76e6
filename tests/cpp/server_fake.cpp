// server_fake.cpp -- the serving loop (genefer22_b200/csrc/gf_server.cpp) on
// the CPU: a gfs::Devices whose pools and checkers are oracle transforms
// (oracle/gf_oracle.c, the restated transformCPUi32).  Test infrastructure:
// built with the loop's own sources into tests/cpp/_build/libgfserver_fake.so
// by tests/test_serve_host.py, which drives the same gfc_server_* C ABI as
// libgfcuda.so exports, with no GPU.
//
// Test hooks: gfc_fake_corrupt(b, block) changes one digit of the residue of
// the test of base b after that many blocks (a fault the Gerbicz-Li check
// must flag); gfc_fake_packed(min_n, b_lo) makes bases >= b_lo "packed" from
// size min_n, so that the pool split by base range runs at small n.
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>

#include "../../genefer22_b200/csrc/gf_server.h"

extern "C" {
void *gfo_create(uint32_t b, uint32_t n, size_t num_regs);
void gfo_destroy(void *h);
void gfo_set(void *h, uint32_t a);
void gfo_square_dup(void *h, int dup);
void gfo_init_multiplicand(void *h, size_t src);
void gfo_mul(void *h);
void gfo_copy(void *h, size_t dst, size_t src);
void gfo_get_zi(const void *h, int32_t *zi);
void gfo_set_zi(void *h, const int32_t *zi);
void gfo_balance(int32_t *d, size_t size, uint32_t base);
}

namespace {

thread_local std::string g_err;
std::mutex g_hook_mu;
uint32_t g_corrupt_b = 0, g_corrupt_block = 0;
uint32_t g_packed_min_n = 19, g_packed_b_lo = 0xffffffffu;

struct Oracle
{
	void *h = nullptr;
	uint32_t b = 0;
	size_t N = 0;
	Oracle(uint32_t b_, uint32_t n) : h(gfo_create(b_, n, 4)), b(b_), N(size_t(1) << n)
	{
		if (h == nullptr) throw gfs::Error{ GFC_ERR_ARG, "oracle: gfo_create failed" };
	}
	~Oracle() { gfo_destroy(h); }
	Oracle(const Oracle &) = delete;
	Oracle &operator=(const Oracle &) = delete;
	void get(size_t reg, int32_t *out)
	{
		if (reg == 0) { gfo_get_zi(h, out); return; }
		gfo_copy(h, 3, 0); gfo_copy(h, 0, reg); gfo_get_zi(h, out); gfo_copy(h, 0, 3);
	}
	void put(size_t reg, const int32_t *in)
	{
		std::vector<int32_t> v(in, in + N);
		gfo_balance(v.data(), N, b);
		if (reg == 0) { gfo_set_zi(h, v.data()); return; }
		gfo_copy(h, 3, 0); gfo_set_zi(h, v.data()); gfo_copy(h, reg, 0); gfo_copy(h, 0, 3);
	}
	void mul_by_reg1() { gfo_init_multiplicand(h, 1); gfo_mul(h); }   // r0 = r0 r1
};

bool bit(const std::vector<uint32_t> &w, uint64_t i) { return ((w[i >> 5] >> (i & 31)) & 1u) != 0; }

class FakePool : public gfs::PoolDev
{
public:
	FakePool(uint32_t n, size_t cap, uint32_t B, uint64_t max_bits) : n_(n), B_(B), max_bits_(max_bits), slots_(cap) {}
	~FakePool() override
	{
		for (int32_t *p : bufs_) std::free(p);
	}
	int plan() const override { return 0; }
	void admit(size_t slot, uint32_t b, const uint32_t *words, uint64_t nbits) override
	{
		// the engine's reserved exponent room (gfc_batch_admit refuses longer exponents)
		if ((nbits == 0) || (nbits > max_bits_)) throw gfs::Error{ GFC_ERR_ARG, "admit: need 1 <= nbits <= the reserved bits" };
		Slot &s = slots_[slot];
		s.o.reset(new Oracle(b, n_));
		gfo_set(s.o->h, 1);
		gfo_copy(s.o->h, 1, 0);
		s.words.assign(words, words + (nbits + 31) / 32);
		s.pos = static_cast<int64_t>(nbits) - 1;
		s.blocks = 0;
	}
	// The graph's work for every slot with bits left: d <- d x, then B squarings.
	void launch_block() override
	{
		for (Slot &s : slots_)
		{
			if (!s.o || (s.pos < 0)) continue;
			void *h = s.o->h;
			gfo_copy(h, 2, 0);
			s.o->mul_by_reg1();
			gfo_copy(h, 1, 0);
			gfo_copy(h, 0, 2);
			for (uint32_t j = 0; (j < B_) && (s.pos >= 0); ++j, --s.pos) gfo_square_dup(h, bit(s.words, uint64_t(s.pos)) ? 1 : 0);
			++s.blocks;
			std::lock_guard<std::mutex> l(g_hook_mu);
			if ((s.o->b == g_corrupt_b) && (s.blocks == g_corrupt_block))
			{
				std::vector<int32_t> d(s.o->N);
				gfo_get_zi(h, d.data());
				d[5] = (d[5] < static_cast<int32_t>(s.o->b / 2)) ? d[5] + 1 : d[5] - 1;
				gfo_set_zi(h, d.data());
			}
		}
	}
	bool block_done() override { return true; }
	void read(size_t slot, int32_t *x, int32_t *d) override
	{
		slots_[slot].o->get(0, x);
		slots_[slot].o->get(1, d);
	}
	bool read_done(size_t) override { return true; }
	int32_t *host_buffer(size_t count) override
	{
		int32_t *p = static_cast<int32_t *>(std::calloc(count, sizeof(int32_t)));
		bufs_.push_back(p);
		return p;
	}

private:
	struct Slot
	{
		std::unique_ptr<Oracle> o;
		std::vector<uint32_t> words;
		int64_t pos = -1;
		uint32_t blocks = 0;
	};
	uint32_t n_, B_;
	uint64_t max_bits_;
	std::vector<Slot> slots_;
	std::vector<int32_t *> bufs_;
};

// genefer::GL (src/genefer.h:557-615) on each item's own oracle transform.
class FakeCheck : public gfs::CheckDev
{
public:
	FakeCheck(uint32_t n, uint32_t B) : n_(n), B_(B) {}
	void start(const std::vector<gfs::CheckItem> &items) override
	{
		ok_.clear();
		for (const gfs::CheckItem &it : items)
		{
			Oracle o(it.b, n_);
			o.put(1, it.d);
			o.put(0, it.x);
			o.mul_by_reg1();                                      // d(t+1) = x d(t)
			gfo_copy(o.h, 2, 0);
			gfo_copy(o.h, 0, 1);
			for (uint32_t j = 0; j < B_; ++j) gfo_square_dup(o.h, 0);   // d(t)^(2^B)
			gfo_copy(o.h, 1, 0);
			gfo_set(o.h, 1);
			for (uint64_t i = it.res_bits; i-- > 0;) gfo_square_dup(o.h, bit(it.res, i) ? 1 : 0);   // 2^res
			o.mul_by_reg1();
			std::vector<int32_t> a(o.N), c(o.N);
			o.get(0, a.data());
			o.get(2, c.data());
			gfc_gint_unbalance(a.data(), o.N, it.b);
			gfc_gint_unbalance(c.data(), o.N, it.b);
			ok_.push_back(gfc_gint_hash64(a.data(), o.N) == gfc_gint_hash64(c.data(), o.N));
		}
	}
	bool done() override { return true; }
	void results(std::vector<bool> &ok) override { ok = ok_; }

private:
	uint32_t n_, B_;
	std::vector<bool> ok_;
};

class FakeDevices : public gfs::Devices
{
public:
	gfs::PoolDev *open_pool(uint32_t n, size_t capacity, uint32_t, uint32_t B, uint64_t max_bits, bool) override
	{
		return new FakePool(n, capacity, B, max_bits);
	}
	gfs::CheckDev *open_check(uint32_t n, size_t, uint32_t B) override { return new FakeCheck(n, B); }
	bool valid(uint32_t b, uint32_t) override { return (b >= 8) && (b < (1u << 31)); }
	bool packed_range(uint32_t b, uint32_t) override
	{
		std::lock_guard<std::mutex> l(g_hook_mu);
		return b >= g_packed_b_lo;
	}
	void pretune(uint32_t, size_t, uint32_t) override {}
	uint32_t packed_pool_min_n() const override
	{
		std::lock_guard<std::mutex> l(g_hook_mu);
		return g_packed_min_n;
	}
};

}  // namespace

namespace gfs {
std::unique_ptr<Devices> make_devices(const gfc_server_config &) { return std::unique_ptr<Devices>(new FakeDevices()); }
}  // namespace gfs

void gfc_internal_set_error(const char *msg) { g_err = (msg != nullptr) ? msg : ""; }

#define FAKE_API extern "C" __attribute__((visibility("default")))

FAKE_API const char *gfc_last_error(void) { return g_err.c_str(); }

FAKE_API void gfc_fake_corrupt(uint32_t b, uint32_t block)
{
	std::lock_guard<std::mutex> l(g_hook_mu);
	g_corrupt_b = b;
	g_corrupt_block = block;
}

FAKE_API void gfc_fake_packed(uint32_t min_n, uint32_t b_lo)
{
	std::lock_guard<std::mutex> l(g_hook_mu);
	g_packed_min_n = min_n;
	g_packed_b_lo = b_lo;
}
