// gf_server_cuda.cpp -- the serving loop's device layer over the engine's
// batches (gfs::make_devices for libgfcuda.so).
//
// A pool is a reserved batch (gfc_batch_reserve) whose block is one CUDA
// graph; its completion is a CUDA event the dispatcher polls.  Admission
// (gfc_batch_admit) and the read-back of finished residues
// (gfc_batch_get_async into pinned buffers) are enqueued on the pool's stream
// without synchronising, so no pool's admission stalls another pool's graph.
// A checker is a reserved batch that runs genefer's Gerbicz-Li check
// (src/genefer.h:557-615) for several finished tests of one size at once.
#include <cuda_runtime.h>

#include <cstring>
#include <map>
#include <mutex>
#include <tuple>

#include "gf_server.h"

void *gfc_internal_pinned_get(size_t bytes);
void gfc_internal_pinned_put(void *p);
void gfc_internal_retain(bool on, size_t bytes);

namespace gfs {

namespace {

void ck(int rc, const char *what)
{
	if (rc != GFC_OK) throw Error{ rc, std::string(what) + ": " + gfc_last_error() };
}

void ckc(cudaError_t e, const char *what)
{
	if (e != cudaSuccess) throw Error{ GFC_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e) };
}

bool query(cudaEvent_t e)
{
	const cudaError_t r = cudaEventQuery(e);
	if (r == cudaSuccess) return true;
	if (r == cudaErrorNotReady) return false;
	ckc(r, "cudaEventQuery");
	return false;
}

// Plans chosen by gfc_batch_tune per pool shape: (n, slots, prime set of the
// representative base, packed range).
class TuneCache
{
public:
	void apply(gfc_batch *bt, uint32_t n, size_t cap, uint32_t rep_b)
	{
		// a pool of packed-range bases tunes with packed plans among the
		// candidates, whatever the RNS width of its representative base
		const int packed = gfc_packed_range(rep_b, n);
		const auto key = std::make_tuple(n, cap, packed ? 4 : gfc_width_for(rep_b, n), packed);
		{
			std::lock_guard<std::mutex> l(mu_);
			auto it = plans_.find(key);
			if (it != plans_.end()) { ck(gfc_batch_set_plan(bt, it->second), "set_plan"); return; }
		}
		int32_t best = 0;
		size_t count = 0;
		ck(gfc_batch_tune(bt, 16, 3, nullptr, nullptr, 0, &count, &best), "tune");
		std::lock_guard<std::mutex> l(mu_);
		plans_[key] = best;
	}

private:
	std::mutex mu_;
	std::map<std::tuple<uint32_t, size_t, int, int>, int32_t> plans_;
};

// Pinned host buffers carved from a few large chunks of the library's pinned
// cache (a pool asks for two per slot; a page-locked allocation per buffer
// made opening a wide pool slow, and freeing one waits for the device).
// The owner destroys them after its last copy completed.
class PinnedBuffers
{
public:
	int32_t *get(size_t count)
	{
		const size_t bytes = (count * sizeof(int32_t) + 255) & ~size_t(255);
		if (bytes > left_)
		{
			const size_t chunk = (bytes > (size_t(8) << 20)) ? bytes : (size_t(8) << 20);
			void *p = gfc_internal_pinned_get(chunk);
			if (p == nullptr) throw Error{ GFC_ERR_CUDA, "no page-locked host memory for a pool's buffers" };
			bufs_.push_back(p);
			next_ = static_cast<char *>(p);
			left_ = chunk;
		}
		int32_t *out = reinterpret_cast<int32_t *>(next_);
		next_ += bytes;
		left_ -= bytes;
		return out;
	}
	~PinnedBuffers()
	{
		for (void *p : bufs_) gfc_internal_pinned_put(p);
	}

private:
	std::vector<void *> bufs_;
	char *next_ = nullptr;
	size_t left_ = 0;
};

class CudaPool : public PoolDev
{
public:
	CudaPool(int device, uint32_t n, size_t cap, uint32_t rep_b, uint32_t B, uint64_t max_bits, bool tune, TuneCache &tc)
		: device_(device), B_(B)
	{
		ckc(cudaSetDevice(device), "cudaSetDevice");
		std::vector<uint32_t> bases(cap, rep_b);
		ck(gfc_batch_create(bases.data(), cap, n, 3, device, nullptr, &bt_), "batch_create");
		if (tune) tc.apply(bt_, n, cap, rep_b);
		ck(gfc_batch_reserve(bt_, (max_bits < B) ? B : max_bits), "reserve");
		capture();
		stream_ = static_cast<cudaStream_t>(gfc_batch_stream(bt_));
		ckc(cudaEventCreateWithFlags(&ev_, cudaEventDisableTiming), "cudaEventCreate");
		read_ev_.assign(cap, nullptr);
		for (cudaEvent_t &e : read_ev_) ckc(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
	}

	~CudaPool() override
	{
		cudaSetDevice(device_);
		if (ev_ != nullptr) cudaEventSynchronize(ev_);
		for (cudaEvent_t e : read_ev_) if (e != nullptr) { cudaEventSynchronize(e); cudaEventDestroy(e); }
		if (ev_ != nullptr) cudaEventDestroy(ev_);
		if (g_ != nullptr) gfc_graph_destroy(g_);
		if (bt_ != nullptr) gfc_batch_destroy(bt_);
	}

	int plan() const override { return gfc_batch_plan(bt_); }

	void admit(size_t slot, uint32_t b, const uint32_t *words, uint64_t nbits) override
	{
		ck(gfc_batch_admit(bt_, slot, b, words, nbits), "admit");
	}

	void launch_block() override
	{
		int rc = gfc_graph_launch(g_);
		if (rc == GFC_ERR_STATE)
		{
			// a slot changed prime set under the single-CTA plan: record again
			gfc_graph_destroy(g_);
			g_ = nullptr;
			capture();
			rc = gfc_graph_launch(g_);
		}
		ck(rc, "graph_launch");
		ckc(cudaEventRecord(ev_, stream_), "cudaEventRecord");
	}

	bool block_done() override { return query(ev_); }

	void read(size_t slot, int32_t *x, int32_t *d) override
	{
		ck(gfc_batch_get_async(bt_, slot, 0, x), "get_async");
		ck(gfc_batch_get_async(bt_, slot, 1, d), "get_async");
		ckc(cudaEventRecord(read_ev_[slot], stream_), "cudaEventRecord");
	}

	bool read_done(size_t slot) override { return query(read_ev_[slot]); }

	int32_t *host_buffer(size_t count) override { return pinned_.get(count); }

private:
	// the block: d <- d x, then B squarings with each slot's exponent bits
	void capture()
	{
		ck(gfc_batch_capture_begin(bt_), "capture_begin");
		const int r1 = gfc_batch_gl_step(bt_);
		const int r2 = (r1 == GFC_OK) ? gfc_batch_square_exp(bt_, B_) : r1;
		gfc_graph *g = nullptr;
		const int r3 = gfc_batch_capture_end(bt_, &g);
		ck(r2, "block");
		ck(r3, "capture_end");
		g_ = g;
	}

	int device_;
	uint32_t B_;
	gfc_batch *bt_ = nullptr;
	gfc_graph *g_ = nullptr;
	cudaStream_t stream_ = nullptr;
	cudaEvent_t ev_ = nullptr;
	std::vector<cudaEvent_t> read_ev_;
	PinnedBuffers pinned_;
};

class CudaCheck : public CheckDev
{
public:
	// The check runs from one CUDA graph (recorded here, again after a change
	// of prime set under the single-CTA plan): enqueued call by call it is
	// thousands of launches at large n, whose queue would hold up the
	// dispatcher thread until the device drained it.  Every exponent 2^res
	// is padded to RB bits with leading zeros (squaring 1 keeps 1), so one
	// graph serves every group.
	CudaCheck(int device, uint32_t n, size_t group, uint32_t B)
		: device_(device), N_(size_t(1) << n), group_(group), B_(B), RB_(B + 96)
	{
		ckc(cudaSetDevice(device), "cudaSetDevice");
		std::vector<uint32_t> bases(group, 1024);
		ck(gfc_batch_create(bases.data(), group, n, 3, device, nullptr, &bt_), "batch_create");
		ck(gfc_batch_reserve(bt_, RB_), "reserve");
		stream_ = static_cast<cudaStream_t>(gfc_batch_stream(bt_));
		ckc(cudaEventCreateWithFlags(&ev_, cudaEventDisableTiming), "cudaEventCreate");
		for (auto *v : { &x_, &d_, &a_, &c_ })
			for (size_t i = 0; i < group; ++i) v->push_back(pinned_.get(N_));
		capture();
	}

	~CudaCheck() override
	{
		cudaSetDevice(device_);
		if (ev_ != nullptr) { cudaEventSynchronize(ev_); cudaEventDestroy(ev_); }
		if (g_ != nullptr) gfc_graph_destroy(g_);
		if (bt_ != nullptr) gfc_batch_destroy(bt_);
	}

	// genefer::GL for every item at once (as genefer22_b200.genefer.gl_validate):
	// d(t+1) = x d(t); d(t)^(2^B) 2^res ?= d(t+1) by hash64.
	void start(const std::vector<CheckItem> &items) override
	{
		k_ = items.size();
		b_.clear();
		const std::vector<uint32_t> zero((RB_ + 31) / 32, 0);
		for (size_t i = 0; i < group_; ++i)
		{
			if (i < k_)
			{
				if (items[i].res_bits > RB_) throw Error{ GFC_ERR_ARG, "check: exponent sum longer than the reserved bits" };
				std::vector<uint32_t> w((RB_ + 31) / 32, 0);
				std::copy(items[i].res.begin(), items[i].res.end(), w.begin());
				ck(gfc_batch_admit(bt_, i, items[i].b, w.data(), RB_), "admit");
				std::memcpy(x_[i], items[i].x, N_ * sizeof(int32_t));
				std::memcpy(d_[i], items[i].d, N_ * sizeof(int32_t));
				ck(gfc_batch_set_async(bt_, i, 0, x_[i]), "set_async");
				ck(gfc_batch_set_async(bt_, i, 1, d_[i]), "set_async");
				b_.push_back(items[i].b);
			}
			else ck(gfc_batch_admit(bt_, i, 1024, zero.data(), RB_), "admit");
		}
		int rc = gfc_graph_launch(g_);
		if (rc == GFC_ERR_STATE)
		{
			gfc_graph_destroy(g_);
			g_ = nullptr;
			capture();
			rc = gfc_graph_launch(g_);
		}
		ck(rc, "graph_launch");
		for (size_t i = 0; i < k_; ++i)
		{
			ck(gfc_batch_get_async(bt_, i, 0, a_[i]), "get_async");
			ck(gfc_batch_get_async(bt_, i, 2, c_[i]), "get_async");
		}
		ckc(cudaEventRecord(ev_, stream_), "cudaEventRecord");
	}

	bool done() override { return query(ev_); }

	void results(std::vector<bool> &ok) override
	{
		ok.assign(k_, false);
		for (size_t i = 0; i < k_; ++i)
		{
			gfc_gint_unbalance(a_[i], N_, b_[i]);
			gfc_gint_unbalance(c_[i], N_, b_[i]);
			ok[i] = (gfc_gint_hash64(a_[i], N_) == gfc_gint_hash64(c_[i], N_));
		}
	}

private:
	void capture()
	{
		ck(gfc_batch_capture_begin(bt_), "capture_begin");
		int rc = gfc_batch_init_multiplicand(bt_, 1);
		if (rc == GFC_OK) rc = gfc_batch_mul(bt_, 0);                 // d(t+1) = x d(t)
		if (rc == GFC_OK) rc = gfc_batch_copy(bt_, 2, 0);
		if (rc == GFC_OK) rc = gfc_batch_copy(bt_, 0, 1);
		if (rc == GFC_OK) rc = gfc_batch_square(bt_, 0, B_);          // d(t)^(2^B)
		if (rc == GFC_OK) rc = gfc_batch_copy(bt_, 1, 0);
		if (rc == GFC_OK) rc = gfc_batch_set(bt_, 1);
		if (rc == GFC_OK) rc = gfc_batch_square_exp(bt_, RB_);        // 2^res
		if (rc == GFC_OK) rc = gfc_batch_init_multiplicand(bt_, 1);
		if (rc == GFC_OK) rc = gfc_batch_mul(bt_, 0);
		gfc_graph *g = nullptr;
		const int rc2 = gfc_batch_capture_end(bt_, &g);
		if ((rc != GFC_OK) && (g != nullptr)) gfc_graph_destroy(g);
		ck(rc, "check sequence");
		ck(rc2, "capture_end");
		g_ = g;
	}

	int device_;
	size_t N_, group_;
	uint32_t B_, RB_;
	gfc_batch *bt_ = nullptr;
	gfc_graph *g_ = nullptr;
	cudaStream_t stream_ = nullptr;
	cudaEvent_t ev_ = nullptr;
	size_t k_ = 0;
	std::vector<uint32_t> b_;
	std::vector<int32_t *> x_, d_, a_, c_;
	PinnedBuffers pinned_;
};

class CudaDevices : public Devices
{
public:
	// Freed device and pinned memory stays with the library for the next
	// pools, up to the budget, while the server runs.
	CudaDevices(int device, uint64_t budget) : device_(device) { gfc_internal_retain(true, budget); }
	~CudaDevices() override { gfc_internal_retain(false, 0); }

	PoolDev *open_pool(uint32_t n, size_t capacity, uint32_t rep_b, uint32_t B, uint64_t max_bits, bool tune) override
	{
		return new CudaPool(device_, n, capacity, rep_b, B, max_bits, tune, tune_);
	}

	CheckDev *open_check(uint32_t n, size_t group, uint32_t B) override { return new CudaCheck(device_, n, group, B); }

	bool valid(uint32_t b, uint32_t n) override { return gfc_width_for(b, n) > 0; }
	bool packed_range(uint32_t b, uint32_t n) override { return gfc_packed_range(b, n) == 1; }

	void pretune(uint32_t n, size_t capacity, uint32_t rep_b) override
	{
		ckc(cudaSetDevice(device_), "cudaSetDevice");
		std::vector<uint32_t> bases(capacity, rep_b);
		gfc_batch *bt = nullptr;
		ck(gfc_batch_create(bases.data(), capacity, n, 3, device_, nullptr, &bt), "batch_create");
		try { tune_.apply(bt, n, capacity, rep_b); }
		catch (...) { gfc_batch_destroy(bt); throw; }
		gfc_batch_destroy(bt);
	}

private:
	int device_;
	TuneCache tune_;
};

}  // namespace

std::unique_ptr<Devices> make_devices(const gfc_server_config &cfg)
{
	int ndev = 0;
	ckc(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
	if ((cfg.device < 0) || (cfg.device >= ndev)) throw Error{ GFC_ERR_ARG, "server: no such device" };
	return std::unique_ptr<Devices>(new CudaDevices(cfg.device, cfg.budget_bytes));
}

}  // namespace gfs
