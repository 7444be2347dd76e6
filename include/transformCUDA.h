/*
 * transformCUDA.h -- genefer's `transform` backend on the B200 engine.
 *
 * A drop-in subclass of genefer's abstract `transform` (src/transform.h:42-256)
 * whose members forward to libgfcuda.so (include/gfcuda.h).  Include it from
 * the genefer tree after "transform.h"; link with -lgfcuda (and -lcudart).
 * Failures of the engine raise std::runtime_error, as genefer's OpenCL
 * backend does (src/ocl.h:166-175).
 *
 * Context files: genefer reads the transform's kind only from the first word
 * of a context (src/transformGPU.h:1127-1150).  This backend writes
 * GFC_CONTEXT_KIND there, a value that no transform::EKind enumerator
 * (src/transform.h:45, 0..11) takes, so a context written by the OpenCL build
 * (EKind::NTT2 / NTT3) or a CPU build fails readContext at the kind check,
 * and a context of this backend fails theirs.  The `transform` base still
 * needs an EKind: NTT3 unless the including code defines TRANSFORM_CUDA_KIND
 * (for example after adding `CUDA` to transform::EKind).
 */
#pragma once

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "transform.h"
#include "gfcuda.h"

#ifndef TRANSFORM_CUDA_KIND
#define TRANSFORM_CUDA_KIND NTT3
#endif

class transformCUDA : public transform
{
private:
	gfc_transform *_h = nullptr;
	const size_t _num_regs;

	static void check(const int rc, const char *const what)
	{
		if (rc != GFC_OK) throw std::runtime_error(std::string("transformCUDA::") + what + ": " + gfc_last_error());
	}

	static gfc_transform *make(const uint32_t b, const uint32_t n, const size_t num_regs, const int device)
	{
		gfc_transform *h = nullptr;
		check(gfc_create(b, n, num_regs, device, nullptr, &h), "create");
		return h;
	}

public:
	// transformGPUs constructor (src/transformGPU.h:945-1083): device ordinal and
	// register count as passed by genefer::createTransformGPU (src/genefer.h:96-108).
	transformCUDA(const uint32_t b, const uint32_t n, const size_t device, const size_t num_regs)
		: transform(size_t(1) << n, n, b, EKind::TRANSFORM_CUDA_KIND),
		  _h(make(b, n, num_regs, static_cast<int>(device))), _num_regs(num_regs) {}

	virtual ~transformCUDA() { gfc_destroy(_h); }

	transformCUDA(const transformCUDA &) = delete;
	transformCUDA &operator=(const transformCUDA &) = delete;

	size_t getMemSize() const override { return gfc_get_mem_size(_h); }
	size_t getCacheSize() const override { return gfc_get_cache_size(_h); }

protected:
	void getZi(int32_t *const zi) const override { check(gfc_get_zi(_h, zi), "getZi"); }
	void setZi(const int32_t *const zi) override { check(gfc_set_zi(_h, zi), "setZi"); }

public:
	void set(const uint32_t a) override { check(gfc_set(_h, a), "set"); }
	void squareDup(const bool dup) override { check(gfc_square_dup(_h, dup ? 1 : 0), "squareDup"); }
	void squareMul(const int32_t a) override { check(gfc_square_mul(_h, a), "squareMul"); }
	void initMultiplicand(const size_t src) override { check(gfc_init_multiplicand(_h, src), "initMultiplicand"); }
	void mul() override { check(gfc_mul(_h), "mul"); }
	void copy(const size_t dst, const size_t src) const override { check(gfc_copy(_h, dst, src), "copy"); }

	// Kind word of this backend's context files (see the file comment).
	static constexpr int context_kind = static_cast<int>(GFC_CONTEXT_KIND);

	// readContext / saveContext (src/transformGPU.h:1127-1150): kind, then the
	// registers; num_regs == 0 means every register.
	bool readContext(file &cFile, const size_t nregs) override
	{
		int kind = 0;
		if (!cFile.read(reinterpret_cast<char *>(&kind), sizeof(kind))) return false;
		if (kind != context_kind) return false;
		const size_t num_regs = (nregs != 0) ? nregs : _num_regs;
		std::vector<char> buf(gfc_context_size(_h, num_regs));
		if (!cFile.read(buf.data(), buf.size())) return false;
		return gfc_read_context(_h, buf.data(), buf.size(), num_regs) == GFC_OK;
	}

	void saveContext(file &cFile, const size_t nregs) const override
	{
		const int kind = context_kind;
		if (!cFile.write(reinterpret_cast<const char *>(&kind), sizeof(kind))) return;
		const size_t num_regs = (nregs != 0) ? nregs : _num_regs;
		std::vector<char> buf(gfc_context_size(_h, num_regs));
		check(gfc_save_context(_h, buf.data(), buf.size(), num_regs), "saveContext");
		cFile.write(buf.data(), buf.size());
	}

	// transform::getError (src/transform.h:72): the engine's arithmetic is
	// exact integer arithmetic, so there is no rounding error to report; a carry
	// that does not fit is an exception from the next synchronising call.
	double getError() const override { return 0; }

	// transform::info (src/transform.h:73; the OpenCL backend prints its split,
	// src/transformGPU.h:903-930): the RNS width and kernel plan of this test.
	void info() const override
	{
		unsigned n = 0;
		while ((size_t(1) << n) < getSize()) ++n;
		std::printf("transformCUDA: n = %u, b = %u, %d primes, plan %d\n", n, getB(), gfc_width(_h), gfc_batch_plan(_h));
	}

	// Number of RNS primes (2, 3, or 4 with packed digits) the engine chose for (b, n).
	int width() const { return gfc_width(_h); }
};
