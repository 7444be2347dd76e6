// gf_server.h -- continuous-batching request loop of the modular-squaring
// engine (internal C++ interface; the C ABI is gfc_server_* in
// include/gfcuda.h).
//
// Requests are Fermat PRP tests, or the first k squarings of one: base b,
// size n, exponent bits.  Tests of one size share a pool: `capacity` slots
// of one batch, whose per-block work (the Gerbicz-Li update d <- d x of
// src/genefer.h:529-535, then B squarings of x with each slot's own exponent
// bits) is one CUDA graph replay.  One dispatcher thread drives every pool:
// when a pool's block is done (a CUDA event), slots whose exponent ran out
// are read back (asynchronously), free slots take waiting requests of their
// size (asynchronous admission, no allocation, no synchronisation), and the
// next block is launched.  So requests that arrive while others run are
// admitted as slots free up, and the pools' blocks overlap on the device.
// Finished tests get genefer's Gerbicz-Li check (src/genefer.h:557-615),
// several of one size at once, on a checker batch of their own.
//
// Pools are opened on helper threads while the device-memory budget allows,
// and closed when idle.  The loop reaches the device only through the
// Devices interface below: libgfcuda.so implements it with the engine's
// batches (gf_server_cuda.cpp); a CPU build for the host-logic tests
// implements it with the CPU oracle.
//
// The reference has no counterpart: genefer runs one test per process
// (src/genefer.h:1360-1480).
#pragma once

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/gfcuda.h"

namespace gfs {

// A failure inside the loop or a device layer: a GFC_ERR_* code and a message.
struct Error
{
	int code;
	std::string msg;
};

// One pool's device side: `capacity` slots of size n, block length B.
struct PoolDev
{
	virtual ~PoolDev() {}
	virtual int plan() const = 0;
	// New test in slot `slot`: r_0 = r_1 = 1, exponent words (nbits bits, a
	// multiple of B), base b.  Enqueued; returns at once.
	virtual void admit(size_t slot, uint32_t b, const uint32_t *words, uint64_t nbits) = 0;
	// One block for every slot that has exponent bits left.
	virtual void launch_block() = 0;
	virtual bool block_done() = 0;
	// Registers 0 (x) and 1 (d(t)) of a slot into host buffers of N digits.
	virtual void read(size_t slot, int32_t *x, int32_t *d) = 0;
	virtual bool read_done(size_t slot) = 0;
	// Host buffer of `count` digits that read() may write asynchronously.
	virtual int32_t *host_buffer(size_t count) = 0;
};

// genefer's Gerbicz-Li check for up to `group` finished tests of one size.
struct CheckItem
{
	uint32_t b;
	const int32_t *x, *d;               // residue and d(t), N digits each
	std::vector<uint32_t> res;          // sum of the exponent's B-bit chunks
	uint64_t res_bits;
};

struct CheckDev
{
	virtual ~CheckDev() {}
	virtual void start(const std::vector<CheckItem> &items) = 0;
	virtual bool done() = 0;
	virtual void results(std::vector<bool> &ok) = 0;
};

struct Devices
{
	virtual ~Devices() {}
	// May run on helper threads (several at once) while the dispatcher drives
	// other pools.
	virtual PoolDev *open_pool(uint32_t n, size_t capacity, uint32_t rep_b, uint32_t B, uint64_t max_bits, bool tune) = 0;
	virtual CheckDev *open_check(uint32_t n, size_t group, uint32_t B) = 0;
	// Whether the engine can run base b at size n at all, and whether b is in
	// the packed-digit range (plans 2xx, 3xx).
	virtual bool valid(uint32_t b, uint32_t n) = 0;
	virtual bool packed_range(uint32_t b, uint32_t n) = 0;
	// Tunes (and caches) the plan of a pool shape before the clock matters.
	virtual void pretune(uint32_t n, size_t capacity, uint32_t rep_b) = 0;
	// From this size a base in the packed range gets a pool of packed-range
	// bases only (packed digits are faster there even for pools of one or two
	// tests, measured on one B200); smaller sizes keep one kind of pool, so
	// that requests are not split between two half-full pools.
	virtual uint32_t packed_pool_min_n() const { return 19; }
};

// The device layer of this build: the engine's batches in libgfcuda.so
// (gf_server_cuda.cpp), the CPU oracle in the host-logic test library.
std::unique_ptr<Devices> make_devices(const gfc_server_config &cfg);

// Device bytes the budget counts (the engine's allocations, gf_host.cu).
uint64_t slot_bytes(uint32_t n);
uint64_t table_bytes(uint32_t n);
uint64_t exponent_bytes(uint64_t nbits);
uint32_t default_capacity(uint32_t n);

// Sum of the B-bit chunks of an exponent (the final 2^res of
// genefer::GL, src/genefer.h:583-592), little-endian words.
std::vector<uint32_t> chunk_sum(const uint32_t *words, uint64_t nbits, uint32_t B, uint64_t *res_bits);

class Server
{
public:
	Server(const gfc_server_config &cfg, std::unique_ptr<Devices> dev);
	~Server();

	void pretune(uint32_t n, uint32_t rep_b);
	void submit(uint64_t id, uint32_t b, uint32_t n, const uint32_t *words, uint64_t nbits);
	// Finished tests (checked, when checking is on); waits up to wait_ms for one.
	size_t poll(gfc_completion *out, size_t cap, int wait_ms);
	bool digits(uint64_t id, int32_t *out, size_t size);
	void info(gfc_server_stats *out);
	double clock() const;
	// First failure of the loop (code, message), or code 0.
	int error(std::string &msg);

private:
	struct Req
	{
		uint64_t id;
		uint32_t b, n;
		std::vector<uint32_t> words;
		uint64_t nbits;
		double arrival;
	};
	enum SlotState { FREE, ACTIVE, READING };
	struct Slot
	{
		SlotState state = FREE;
		Req req;
		gfc_completion comp{};
		uint64_t blocks_left = 0;
		int32_t *x = nullptr, *d = nullptr;
	};
	struct Pool
	{
		int pid = 0;
		uint32_t n = 0;
		size_t cap = 0;
		uint64_t bytes = 0;
		bool packed_only = false;
		uint32_t rep_b = 0;
		std::unique_ptr<PoolDev> dev;      // null while a helper thread opens it
		std::vector<Slot> slots;
		bool inflight = false;
		double idle_since = 0;
	};
	struct Finished
	{
		gfc_completion comp;
		std::vector<int32_t> x, d;
		std::vector<uint32_t> res;
		uint64_t res_bits;
	};
	struct Checker
	{
		uint32_t n = 0;
		uint64_t bytes = 0;
		std::unique_ptr<CheckDev> dev;     // null until opened
		bool opening = false, busy = false;
		bool finishing = false;            // a helper thread is computing the group's results
		std::deque<Finished> queue;
		std::vector<Finished> group;
	};

	void loop();
	void step(bool &progress);
	void service_pool(Pool &p, bool &progress);
	void place();
	void service_checkers(bool &progress);
	void finish(gfc_completion c, std::vector<int32_t> canon);
	bool take_budget(uint32_t n, uint64_t bytes);
	void give_budget(uint32_t n, uint64_t bytes);
	void close_idle_pools();
	void opener();
	void fail_loop(int code, const std::string &msg);

	gfc_server_config cfg_;
	std::unique_ptr<Devices> dev_;
	const std::chrono::steady_clock::time_point t0_;

	// submit -> dispatcher
	std::mutex in_mu_;
	std::vector<Req> incoming_;
	uint64_t submitted_ = 0;

	// dispatcher state
	std::map<uint32_t, std::deque<Req>> waiting_;
	std::vector<std::unique_ptr<Pool>> pools_;
	std::map<uint32_t, Checker> checkers_;
	int next_pid_ = 0;
	uint64_t used_ = 0, peak_ = 0;
	std::map<uint32_t, int> tables_;            // pools + checkers holding each size's tables
	uint64_t pools_created_ = 0, blocks_run_ = 0, gl_failures_ = 0;
	double open_s_sum_ = 0, open_s_max_ = 0, step_s_max_ = 0;   // helper-thread opens, longest dispatcher step
	// longest parts of a dispatcher pass: continuations, pools, placing, checks,
	// closing; and of servicing a pool: event query, read-back, admission, block launch
	double phase_max_[9] = { 0, 0, 0, 0, 0, 0, 0, 0, 0 };
	void note_phase(int k, double t0);

	// helper threads: open pools and checkers
	std::mutex op_mu_;
	std::condition_variable op_cv_;
	struct OpenJob
	{
		Pool *pool;            // or null for a checker
		uint32_t n;
		uint64_t max_bits;
	};
	std::deque<OpenJob> open_jobs_;
	std::deque<std::unique_ptr<PoolDev>> close_jobs_;   // closed pools, released by the helper threads
	// Host work of the residues (canonical digits, res64, Gerbicz-Li hashes:
	// seconds at n = 22, 23) runs on the helper threads; what it changes in
	// the dispatcher's state it posts back as continuations, run by the
	// dispatcher at its next pass.
	std::deque<std::function<void()>> host_jobs_;
	std::mutex cont_mu_;
	std::deque<std::function<void()>> continuations_;
	void post_host(std::function<void()> f);
	void post_cont(std::function<void()> f);
	std::vector<std::pair<Pool *, std::unique_ptr<PoolDev>>> opened_pools_;
	std::vector<std::pair<uint32_t, std::unique_ptr<CheckDev>>> opened_checks_;
	std::vector<std::thread> openers_;     // pools of different sizes open in parallel

	// dispatcher -> poll
	std::mutex out_mu_;
	std::condition_variable out_cv_;
	std::deque<gfc_completion> done_;
	std::map<uint64_t, std::vector<int32_t>> digits_;
	uint64_t completed_ = 0;
	int err_code_ = 0;
	std::string err_msg_;

	std::atomic<bool> stop_{ false };
	uint64_t pools_open_ = 0;
	std::thread thread_;
};

}  // namespace gfs
