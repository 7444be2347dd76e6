// gf_server.cpp -- the continuous-batching request loop (gf_server.h).
//
// Plain C++ (no CUDA): the device work goes through gfs::Devices, so the same
// loop runs in libgfcuda.so over the engine and, for the host-logic tests, on
// the CPU over the oracle.
#include "gf_server.h"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <stdexcept>

namespace gfs {

namespace {

constexpr uint32_t NUM_REGS = 3;
constexpr int OPENERS = 4;     // helper threads that open pools and checkers

}  // namespace

// Device bytes of one slot as gfc_batch_create allocates them: registers,
// 3 transform planes, 3 multiplicand planes, segment carries (five values per
// 16 digits), descriptor, test index and position.
uint64_t slot_bytes(uint32_t n)
{
	const uint64_t N = uint64_t(1) << n;
	return NUM_REGS * 4 * N + 12 * N + 12 * N + (N / 16) * 8 * 5 + 1024;
}

// Root tables of size n shared by every batch of that size on a device:
// 16 N words for the prime sets of one digit per coefficient, 8 N for packed
// digits (get_tables, get_tables_packed in gf_host.cu).
uint64_t table_bytes(uint32_t n) { return 24 * 4 * (uint64_t(1) << n); }

uint64_t exponent_bytes(uint64_t nbits) { return 4 * ((((nbits + 31) / 32) + 3) & ~uint64_t(3)); }

// Slots per pool: enough tests per launch to fill the GPU at small n, few at
// large n where one test already fills it (measured on one B200).
uint32_t default_capacity(uint32_t n)
{
	static const uint32_t cap[24] = { 32, 32, 32, 32, 32, 32, 32, 32, 32, 32, 32, 32, 32, 32, 32, 32, 32, 16, 8, 4, 2, 2, 1, 1 };
	return (n < 24) ? cap[n] : 1;
}

std::vector<uint32_t> chunk_sum(const uint32_t *words, uint64_t nbits, uint32_t B, uint64_t *res_bits)
{
	// sum over chunks k of bits [k B, (k + 1) B)
	const uint64_t nch = (nbits + B - 1) / B;
	std::vector<uint32_t> acc((B + 64 + 31) / 32 + 1, 0);
	auto bit = [&](uint64_t i) -> uint32_t { return (i < nbits) ? ((words[i >> 5] >> (i & 31)) & 1u) : 0u; };
	for (uint64_t k = 0; k < nch; ++k)
	{
		uint64_t carry = 0;
		for (size_t w = 0; w < acc.size(); ++w)
		{
			uint32_t v = 0;
			for (uint32_t j = 0; j < 32; ++j)
			{
				const uint64_t pos = uint64_t(w) * 32 + j;
				if (pos < B) v |= bit(k * B + pos) << j;
			}
			const uint64_t s = uint64_t(acc[w]) + v + carry;
			acc[w] = static_cast<uint32_t>(s);
			carry = s >> 32;
		}
	}
	uint64_t bits = 0;
	for (size_t w = acc.size(); w-- > 0;)
		if (acc[w] != 0) { bits = 32 * w + (32 - __builtin_clz(acc[w])); break; }
	*res_bits = (bits == 0) ? 1 : bits;
	acc.resize((*res_bits + 31) / 32);
	return acc;
}

Server::Server(const gfc_server_config &cfg, std::unique_ptr<Devices> dev)
	: cfg_(cfg), dev_(std::move(dev)), t0_(std::chrono::steady_clock::now())
{
	if (cfg_.block == 0) throw Error{ GFC_ERR_ARG, "server: block length must be >= 1" };
	for (int i = 0; i < OPENERS; ++i) openers_.emplace_back([this] { opener(); });
	thread_ = std::thread([this] { loop(); });
}

Server::~Server()
{
	stop_ = true;
	if (thread_.joinable()) thread_.join();
	{
		std::lock_guard<std::mutex> l(op_mu_);
		open_jobs_.clear();
	}
	op_cv_.notify_all();
	for (std::thread &t : openers_)
		if (t.joinable()) t.join();
}

double Server::clock() const
{
	return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
}

void Server::pretune(uint32_t n, uint32_t rep_b)
{
	const uint32_t cap = cfg_.capacity[n < 24 ? n : 23] ? cfg_.capacity[n < 24 ? n : 23] : default_capacity(n);
	dev_->pretune(n, cap, rep_b);
}

void Server::submit(uint64_t id, uint32_t b, uint32_t n, const uint32_t *words, uint64_t nbits)
{
	if ((n < 8) || (n > 23) || (nbits == 0) || (words == nullptr)) throw Error{ GFC_ERR_ARG, "submit: need 8 <= n <= 23 and an exponent" };
	if (!dev_->valid(b, n)) throw Error{ GFC_ERR_RANGE, "submit: (b, n) is outside the engine's exact range" };
	Req r;
	r.id = id; r.b = b; r.n = n; r.nbits = nbits;
	r.words.assign(words, words + (nbits + 31) / 32);
	if (nbits % 32 != 0) r.words.back() &= (uint32_t(1) << (nbits % 32)) - 1;   // bits above the exponent
	std::lock_guard<std::mutex> l(in_mu_);
	r.arrival = clock();
	incoming_.push_back(std::move(r));
	++submitted_;
}

size_t Server::poll(gfc_completion *out, size_t cap, int wait_ms)
{
	std::unique_lock<std::mutex> l(out_mu_);
	if (done_.empty() && (wait_ms > 0) && (err_code_ == 0))
		out_cv_.wait_for(l, std::chrono::milliseconds(wait_ms), [&] { return !done_.empty() || (err_code_ != 0); });
	size_t k = 0;
	while ((k < cap) && !done_.empty()) { out[k++] = done_.front(); done_.pop_front(); }
	return k;
}

bool Server::digits(uint64_t id, int32_t *out, size_t size)
{
	std::lock_guard<std::mutex> l(out_mu_);
	auto it = digits_.find(id);
	if ((it == digits_.end()) || (it->second.size() != size)) return false;
	std::memcpy(out, it->second.data(), size * sizeof(int32_t));
	digits_.erase(it);
	return true;
}

void Server::info(gfc_server_stats *out)
{
	std::memset(out, 0, sizeof(*out));
	{
		std::lock_guard<std::mutex> l(in_mu_);
		out->submitted = submitted_;
	}
	std::lock_guard<std::mutex> l(out_mu_);
	out->completed = completed_;
	out->pools_created = pools_created_;
	out->blocks_run = blocks_run_;
	out->peak_bytes = peak_;
	out->used_bytes = used_;
	out->budget_bytes = cfg_.budget_bytes;
	out->gl_failures = gl_failures_;
	out->open_s_sum = open_s_sum_;
	out->open_s_max = open_s_max_;
	out->step_s_max = step_s_max_;
	for (int k = 0; k < 9; ++k) out->phase_s_max[k] = phase_max_[k];
	out->pools_open = pools_open_;
}

int Server::error(std::string &msg)
{
	std::lock_guard<std::mutex> l(out_mu_);
	msg = err_msg_;
	return err_code_;
}

void Server::fail_loop(int code, const std::string &msg)
{
	{
		std::lock_guard<std::mutex> l(out_mu_);
		if (err_code_ == 0) { err_code_ = code; err_msg_ = msg; }
	}
	out_cv_.notify_all();
}

// ------------------------------------------------------------------ budget

bool Server::take_budget(uint32_t n, uint64_t bytes)
{
	const uint64_t total = bytes + ((tables_[n] > 0) ? 0 : table_bytes(n));
	if (used_ + total > cfg_.budget_bytes) return false;
	std::lock_guard<std::mutex> l(out_mu_);
	used_ += total;
	peak_ = std::max(peak_, used_);
	tables_[n]++;
	return true;
}

void Server::give_budget(uint32_t n, uint64_t bytes)
{
	std::lock_guard<std::mutex> l(out_mu_);
	tables_[n]--;
	used_ -= bytes + ((tables_[n] == 0) ? table_bytes(n) : 0);
}

// ------------------------------------------------------------------ helper thread

void Server::opener()
{
	for (;;)
	{
		OpenJob job;
		std::unique_ptr<PoolDev> closing;
		std::function<void()> host;
		{
			std::unique_lock<std::mutex> l(op_mu_);
			op_cv_.wait(l, [&] { return !open_jobs_.empty() || !close_jobs_.empty() || !host_jobs_.empty() || stop_; });
			if (!host_jobs_.empty())
			{
				host = std::move(host_jobs_.front());
				host_jobs_.pop_front();
			}
			else if (!close_jobs_.empty())
			{
				closing = std::move(close_jobs_.front());
				close_jobs_.pop_front();
			}
			else
			{
				if (open_jobs_.empty()) return;
				job = open_jobs_.front();
				open_jobs_.pop_front();
			}
		}
		if (host)
		{
			try { host(); }
			catch (const Error &e) { fail_loop(e.code, e.msg); }
			catch (const std::exception &e) { fail_loop(GFC_ERR_CUDA, e.what()); }
			continue;
		}
		if (closing)
		{
			// releasing a pool frees device memory, which waits for the whole
			// device: done here, not on the dispatcher thread
			try { closing.reset(); }
			catch (...) { }
			continue;
		}
		const double t_open = clock();
		try
		{
			if (job.pool != nullptr)
			{
				Pool &p = *job.pool;
				std::unique_ptr<PoolDev> d(dev_->open_pool(p.n, p.cap, p.rep_b, cfg_.block, job.max_bits, cfg_.tune != 0));
				for (Slot &s : p.slots)
				{
					s.x = d->host_buffer(size_t(1) << p.n);
					s.d = d->host_buffer(size_t(1) << p.n);
				}
				std::lock_guard<std::mutex> l(op_mu_);
				opened_pools_.emplace_back(job.pool, std::move(d));
			}
			else
			{
				std::unique_ptr<CheckDev> c(dev_->open_check(job.n, cfg_.validate_group, cfg_.block));
				std::lock_guard<std::mutex> l(op_mu_);
				opened_checks_.emplace_back(job.n, std::move(c));
			}
			{
				const double dt = clock() - t_open;
				std::lock_guard<std::mutex> l(out_mu_);
				open_s_sum_ += dt;
				open_s_max_ = std::max(open_s_max_, dt);
			}
		}
		catch (const Error &e) { fail_loop(e.code, e.msg); }
		catch (const std::exception &e) { fail_loop(GFC_ERR_CUDA, e.what()); }
	}
}

void Server::post_host(std::function<void()> f)
{
	{
		std::lock_guard<std::mutex> l(op_mu_);
		host_jobs_.push_back(std::move(f));
	}
	op_cv_.notify_one();
}

void Server::post_cont(std::function<void()> f)
{
	std::lock_guard<std::mutex> l(cont_mu_);
	continuations_.push_back(std::move(f));
}

// ------------------------------------------------------------------ dispatcher

void Server::loop()
{
	try
	{
		while (!stop_)
		{
			bool progress = false;
			const double t_step = clock();
			step(progress);
			const double dt = clock() - t_step;
			if (dt > step_s_max_)
			{
				std::lock_guard<std::mutex> l(out_mu_);
				step_s_max_ = dt;
			}
			if (!progress) std::this_thread::sleep_for(std::chrono::microseconds(50));
		}
	}
	catch (const Error &e) { fail_loop(e.code, e.msg); }
	catch (const std::exception &e) { fail_loop(GFC_ERR_CUDA, e.what()); }
	// drain: the device work of every pool ends before the pools go
	try
	{
		for (auto &p : pools_)
			if (p->dev && p->inflight)
				while (!p->dev->block_done()) std::this_thread::sleep_for(std::chrono::microseconds(100));
		for (auto &c : checkers_)
			if (c.second.dev && c.second.busy)
				while (!c.second.dev->done()) std::this_thread::sleep_for(std::chrono::microseconds(100));
	}
	catch (...) { }
	{
		// the helper thread finishes its current open (they point into pools_)
		// and exits, also when the loop ended on a failure rather than on stop
		std::unique_lock<std::mutex> l(op_mu_);
		open_jobs_.clear();
		stop_ = true;
	}
	// (helper threads release queued closed pools before they exit)
	op_cv_.notify_all();
	for (std::thread &t : openers_)
		if (t.joinable()) t.join();
	opened_pools_.clear();
	opened_checks_.clear();
	pools_.clear();
	checkers_.clear();
}

void Server::step(bool &progress)
{
	{
		std::lock_guard<std::mutex> l(out_mu_);
		if (err_code_ != 0) throw Error{ err_code_, err_msg_ };
	}
	{
		std::lock_guard<std::mutex> l(in_mu_);
		for (Req &r : incoming_)
		{
			waiting_[r.n].push_back(std::move(r));
			progress = true;
		}
		incoming_.clear();
	}
	{
		std::lock_guard<std::mutex> l(op_mu_);
		for (auto &o : opened_pools_) { o.first->dev = std::move(o.second); progress = true; }
		opened_pools_.clear();
		for (auto &o : opened_checks_)
		{
			Checker &c = checkers_[o.first];
			c.dev = std::move(o.second);
			c.opening = false;
			progress = true;
		}
		opened_checks_.clear();
	}
	double t = clock();
	auto lap = [&](int k) {
		const double now = clock();
		if (now - t > phase_max_[k])
		{
			std::lock_guard<std::mutex> l(out_mu_);
			phase_max_[k] = now - t;
		}
		t = now;
	};
	{
		std::deque<std::function<void()>> conts;
		{
			std::lock_guard<std::mutex> l(cont_mu_);
			conts.swap(continuations_);
		}
		for (auto &f : conts) { f(); progress = true; }
	}
	lap(0);
	for (auto &p : pools_)
		if (p->dev) service_pool(*p, progress);
	lap(1);
	place();
	lap(2);
	service_checkers(progress);
	lap(3);
	close_idle_pools();
	lap(4);
}

void Server::note_phase(int k, double t0)
{
	const double dt = clock() - t0;
	if (dt > phase_max_[k])
	{
		std::lock_guard<std::mutex> l(out_mu_);
		phase_max_[k] = dt;
	}
}

void Server::service_pool(Pool &p, bool &progress)
{
	const double now = clock();
	if (p.inflight)
	{
		const double tq = clock();
		const bool done = p.dev->block_done();
		note_phase(5, tq);
		if (!done) return;
		p.inflight = false;
		progress = true;
		{
			std::lock_guard<std::mutex> l(out_mu_);
			++blocks_run_;
		}
		for (size_t i = 0; i < p.cap; ++i)
		{
			Slot &s = p.slots[i];
			if ((s.state == ACTIVE) && (--s.blocks_left == 0))
			{
				const double tr = clock();
				p.dev->read(i, s.x, s.d);
				note_phase(6, tr);
				s.state = READING;
			}
		}
	}
	// finished tests whose residues have reached the host
	for (size_t i = 0; i < p.cap; ++i)
	{
		Slot &s = p.slots[i];
		if ((s.state != READING) || !p.dev->read_done(i)) continue;
		// the residue is on the host: copy it out of the slot's buffers, free the
		// slot, and leave the canonical digits, res64 and the check's inputs to a
		// helper thread
		const size_t N = size_t(1) << p.n;
		const bool check = (cfg_.validate_group > 0);
		auto f = std::make_shared<Finished>();
		f->comp = s.comp;
		f->comp.residue_at = clock();
		f->x.assign(s.x, s.x + N);
		if (check)
		{
			f->d.assign(s.d, s.d + N);
			f->res = chunk_sum(s.req.words.data(), s.req.nbits, cfg_.block, &f->res_bits);
		}
		const uint32_t b = s.req.b, n = p.n;
		post_host([this, f, b, n, check]() {
			auto canon = std::make_shared<std::vector<int32_t>>(f->x);
			gfc_gint_unbalance(canon->data(), canon->size(), b);
			uint64_t r64 = 0, o64 = 0;
			f->comp.is_prp = gfc_gint_is_one(canon->data(), canon->size(), b, &r64, &o64);
			f->comp.res64 = r64;
			f->comp.old64 = o64;
			post_cont([this, f, canon, n, check]() {
				if (check)
				{
					if (cfg_.keep_digits)
					{
						std::lock_guard<std::mutex> l(out_mu_);
						digits_[f->comp.id] = std::move(*canon);
					}
					checkers_[n].n = n;
					checkers_[n].queue.push_back(std::move(*f));
				}
				else finish(f->comp, std::move(*canon));
			});
		});
		s.state = FREE;
		s.req = Req();
		progress = true;
	}
	// admission: waiting requests of this size into free slots
	auto &q = waiting_[p.n];
	for (size_t i = 0; (i < p.cap) && !q.empty(); ++i)
	{
		Slot &s = p.slots[i];
		if (s.state != FREE) continue;
		auto it = q.begin();
		if (p.packed_only)
			it = std::find_if(q.begin(), q.end(), [&](const Req &r) { return dev_->packed_range(r.b, r.n); });
		if (it == q.end()) break;
		s.req = std::move(*it);
		q.erase(it);
		const uint64_t pad = ((s.req.nbits + cfg_.block - 1) / cfg_.block) * cfg_.block;
		std::vector<uint32_t> w((pad + 31) / 32, 0);
		std::copy(s.req.words.begin(), s.req.words.end(), w.begin());
		const double ta = clock();
		p.dev->admit(i, s.req.b, w.data(), pad);
		note_phase(7, ta);
		s.blocks_left = pad / cfg_.block;
		s.state = ACTIVE;
		std::memset(&s.comp, 0, sizeof(s.comp));
		s.comp.id = s.req.id; s.comp.b = s.req.b; s.comp.n = s.req.n; s.comp.nbits = s.req.nbits;
		s.comp.arrival = s.req.arrival;
		s.comp.admitted = clock();
		s.comp.validated_at = -1;
		s.comp.gl_ok = -1;
		s.comp.pool = p.pid;
		s.comp.slot = static_cast<int32_t>(i);
		s.comp.plan = p.dev->plan();
		progress = true;
	}
	bool active = false;
	for (const Slot &s : p.slots) active |= (s.state == ACTIVE);
	if (active)
	{
		const double tl = clock();
		p.dev->launch_block();
		note_phase(8, tl);
		p.inflight = true;
		progress = true;
		p.idle_since = now;
	}
	else
	{
		bool reading = false;
		for (const Slot &s : p.slots) reading |= (s.state == READING);
		if (reading) p.idle_since = now;
	}
}

// Opens pools for waiting requests while the budget allows (a pool opened at
// n >= 19 for a base in the packed range tunes with that base, so packed
// plans are candidates, and takes only such bases; any other pool takes every
// base).  The slots of pools still being opened count as free.
void Server::place()
{
	for (auto &kv : waiting_)
	{
		const uint32_t n = kv.first;
		const auto &q = kv.second;
		if (q.empty()) continue;
		size_t any_w = 0, pk_w = 0;
		uint32_t pk_rep = 0;
		for (const Req &r : q)
		{
			if ((n >= dev_->packed_pool_min_n()) && dev_->packed_range(r.b, n)) { if (pk_w++ == 0) pk_rep = r.b; }
			else ++any_w;
		}
		size_t free_any = 0, free_pk = 0;
		for (const auto &p : pools_)
		{
			if (p->n != n) continue;
			size_t f = 0;
			for (const Slot &s : p->slots) f += (s.state == FREE);
			(p->packed_only ? free_pk : free_any) += f;
		}
		for (;;)
		{
			uint32_t rep;
			bool pk;
			if (free_any < any_w) { rep = 1024; pk = false; }
			else if (free_pk + (free_any - any_w) < pk_w) { rep = pk_rep; pk = true; }
			else break;
			const uint32_t cap = (cfg_.capacity[n] != 0) ? cfg_.capacity[n] : default_capacity(n);
			// every slot can hold the longest exponent of its size: b < 2^31 gives
			// b^(2^n) fewer than 31 2^n bits, padded to whole blocks
			const uint64_t mb = (uint64_t(31) << n) + cfg_.block;
			const uint64_t bytes = cap * (slot_bytes(n) + exponent_bytes(mb));
			// the first pool of a size also brings the size's checker
			const bool need_check = (cfg_.validate_group > 0) && (checkers_.count(n) == 0 || checkers_[n].bytes == 0);
			const uint64_t cbytes = need_check ? cfg_.validate_group * (slot_bytes(n) + exponent_bytes(cfg_.block + 96)) : 0;
			if (!take_budget(n, bytes + cbytes))
			{
				bool any_pool = false;
				for (const auto &p : pools_) any_pool |= (p->n == n);
				if (!any_pool && pools_.empty())
					throw Error{ GFC_ERR_ARG, "server: the memory budget cannot hold one pool of this size" };
				break;
			}
			auto p = std::make_unique<Pool>();
			p->pid = next_pid_++;
			p->n = n;
			p->cap = cap;
			p->bytes = bytes;
			p->packed_only = pk;
			p->rep_b = rep;
			p->slots.resize(cap);
			p->idle_since = clock();
			{
				std::lock_guard<std::mutex> l(out_mu_);
				++pools_created_;
				++pools_open_;
			}
			{
				std::lock_guard<std::mutex> l(op_mu_);
				open_jobs_.push_back({ p.get(), n, mb });
				if (need_check)
				{
					tables_[n]++;            // the checker holds the size's tables too
					Checker &c = checkers_[n];
					c.n = n;
					c.bytes = cbytes;
					c.opening = true;
					open_jobs_.push_back({ nullptr, n, 0 });
				}
			}
			op_cv_.notify_all();
			(pk ? free_pk : free_any) += cap;
			pools_.push_back(std::move(p));
		}
	}
}

void Server::service_checkers(bool &progress)
{
	for (auto &kv : checkers_)
	{
		Checker &c = kv.second;
		if (!c.dev) continue;
		if (c.busy)
		{
			if (c.finishing || !c.dev->done()) continue;
			// the hashes of the group's residues on a helper thread; the checker
			// stays busy until its continuation has recorded them
			c.finishing = true;
			Checker *cp = &c;
			post_host([this, cp]() {
				auto ok = std::make_shared<std::vector<bool>>();
				cp->dev->results(*ok);
				post_cont([this, cp, ok]() {
					const double now = clock();
					for (size_t i = 0; i < cp->group.size(); ++i)
					{
						gfc_completion comp = cp->group[i].comp;
						comp.gl_ok = (*ok)[i] ? 1 : 0;
						comp.validated_at = now;
						if (!(*ok)[i])
						{
							std::lock_guard<std::mutex> l(out_mu_);
							++gl_failures_;
						}
						finish(comp, {});
					}
					cp->group.clear();
					cp->busy = false;
					cp->finishing = false;
				});
			});
			progress = true;
			continue;
		}
		if (c.queue.empty()) continue;
		const size_t k = std::min<size_t>(c.queue.size(), cfg_.validate_group);
		std::vector<CheckItem> items;
		for (size_t i = 0; i < k; ++i)
		{
			c.group.push_back(std::move(c.queue.front()));
			c.queue.pop_front();
		}
		for (const Finished &f : c.group) items.push_back({ f.comp.b, f.x.data(), f.d.data(), f.res, f.res_bits });
		c.dev->start(items);
		c.busy = true;
		progress = true;
	}
}

void Server::finish(gfc_completion c, std::vector<int32_t> canon)
{
	{
		std::lock_guard<std::mutex> l(out_mu_);
		if (cfg_.keep_digits && !canon.empty()) digits_[c.id] = std::move(canon);
		done_.push_back(c);
		++completed_;
	}
	out_cv_.notify_all();
}

// A pool with no test in it and nothing waiting for its size closes after
// idle_close_s, or at once when a waiting request of another size cannot get
// a pool for lack of budget.  Closing frees device memory.
void Server::close_idle_pools()
{
	const double now = clock();
	bool starved = false;
	for (const auto &kv : waiting_)
	{
		if (kv.second.empty()) continue;
		bool has = false;
		for (const auto &p : pools_) has |= (p->n == kv.first);
		starved |= !has;
	}
	for (size_t i = 0; i < pools_.size();)
	{
		Pool &p = *pools_[i];
		bool busy = p.inflight || !p.dev;
		for (const Slot &s : p.slots) busy |= (s.state != FREE);
		const bool wanted = !waiting_[p.n].empty();
		if (!busy && !wanted && (starved || (now - p.idle_since > cfg_.idle_close_s)))
		{
			give_budget(p.n, p.bytes);
			{
				std::lock_guard<std::mutex> l(op_mu_);
				close_jobs_.push_back(std::move(p.dev));
			}
			op_cv_.notify_all();
			pools_.erase(pools_.begin() + static_cast<std::ptrdiff_t>(i));
			std::lock_guard<std::mutex> l(out_mu_);
			--pools_open_;
			continue;
		}
		++i;
	}
}

}  // namespace gfs

// ------------------------------------------------------------------ C ABI (include/gfcuda.h)

void gfc_internal_set_error(const char *msg);   // message for gfc_last_error on this thread

#define GFC_API extern "C" __attribute__((visibility("default")))

struct gfc_server
{
	std::unique_ptr<gfs::Server> s;
};

namespace {

template <class F>
int sguard(F &&f)
{
	try
	{
		f();
		return GFC_OK;
	}
	catch (const gfs::Error &e)
	{
		gfc_internal_set_error(e.msg.c_str());
		return e.code;
	}
	catch (const std::exception &e)
	{
		gfc_internal_set_error(e.what());
		return GFC_ERR_CUDA;
	}
}

void null_check(const void *p)
{
	if (p == nullptr) throw gfs::Error{ GFC_ERR_ARG, "null handle or pointer" };
}

}  // namespace

GFC_API void gfc_server_default_config(gfc_server_config *cfg)
{
	if (cfg == nullptr) return;
	std::memset(cfg, 0, sizeof(*cfg));
	cfg->block = 1000;
	cfg->validate_group = 4;
	cfg->budget_bytes = uint64_t(80) * 1000 * 1000 * 1000;
	cfg->device = 0;
	cfg->tune = 1;
	cfg->keep_digits = 0;
	cfg->idle_close_s = 10.0;
}

GFC_API int gfc_server_create(const gfc_server_config *cfg, gfc_server **out)
{
	return sguard([&] {
		null_check(cfg); null_check(out);
		*out = nullptr;
		std::unique_ptr<gfc_server> s(new gfc_server());
		s->s.reset(new gfs::Server(*cfg, gfs::make_devices(*cfg)));
		*out = s.release();
	});
}

GFC_API int gfc_server_pretune(gfc_server *s, uint32_t n, uint32_t rep_b)
{
	return sguard([&] {
		null_check(s);
		if ((n < 8) || (n > 23)) throw gfs::Error{ GFC_ERR_ARG, "pretune: need 8 <= n <= 23" };
		s->s->pretune(n, rep_b);
	});
}

GFC_API int gfc_server_submit(gfc_server *s, uint64_t id, uint32_t b, uint32_t n, const uint32_t *words, uint64_t nbits)
{
	return sguard([&] { null_check(s); s->s->submit(id, b, n, words, nbits); });
}

GFC_API int gfc_server_poll(gfc_server *s, gfc_completion *out, size_t cap, size_t *got, int32_t wait_ms)
{
	return sguard([&] {
		null_check(s); null_check(got);
		if ((out == nullptr) && (cap != 0)) throw gfs::Error{ GFC_ERR_ARG, "poll: null output" };
		*got = s->s->poll(out, cap, wait_ms);
		std::string msg;
		const int code = s->s->error(msg);
		if (code != 0) throw gfs::Error{ code, "server loop: " + msg };
	});
}

GFC_API int gfc_server_digits(gfc_server *s, uint64_t id, int32_t *out, size_t size)
{
	return sguard([&] {
		null_check(s); null_check(out);
		if (!s->s->digits(id, out, size)) throw gfs::Error{ GFC_ERR_STATE, "digits: no kept residue of this id and size" };
	});
}

GFC_API int gfc_server_get_stats(gfc_server *s, gfc_server_stats *out)
{
	return sguard([&] { null_check(s); null_check(out); s->s->info(out); });
}

GFC_API double gfc_server_clock(const gfc_server *s) { return (s == nullptr) ? 0.0 : s->s->clock(); }

GFC_API void gfc_server_destroy(gfc_server *s) { delete s; }

GFC_API uint64_t gfc_server_slot_bytes(uint32_t n, uint64_t max_bits)
{
	return ((n < 8) || (n > 23)) ? 0 : gfs::slot_bytes(n) + gfs::exponent_bytes(max_bits);
}

GFC_API uint64_t gfc_server_table_bytes(uint32_t n) { return ((n < 8) || (n > 23)) ? 0 : gfs::table_bytes(n); }

GFC_API uint32_t gfc_server_default_capacity(uint32_t n) { return gfs::default_capacity(n); }
