/*
 * ref_harness.cpp -- C ABI over the REFERENCE's own CPU transforms (test
 * infrastructure and CPU baseline only; never part of the product path).
 *
 * Compiled by oracle/Makefile together with the reference translation units
 * src/transform_{i32,sse2,sse4,avx,fma,512}.cpp, read where they lie in the
 * reference tree, into oracle/_ref/libgfref.so.  Every entry point forwards
 * to the reference's public `transform` API (src/transform.h:58-70,
 * :122-193, :228-246); nothing here re-implements arithmetic.
 */
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <unistd.h>

#include "transform.h"

#define REF_API extern "C" __attribute__((visibility("default")))

namespace
{
struct ref_handle
{
	transform *t;
	gint *g;
	uint32_t b, n;
	std::string ttype;
};
thread_local std::string g_last_error;
}

REF_API const char *ref_last_error() { return g_last_error.c_str(); }

/* transform::create_cpu (src/transform.h:122-193): impl is "i32", "512",
   "fma", "avx", "sse4", "sse2" or "" (best available). */
REF_API void *ref_create(uint32_t b, uint32_t n, size_t num_regs, const char *impl, size_t num_threads, int check_error)
{
	try
	{
		ref_handle *h = new ref_handle();
		h->b = b; h->n = n;
		h->t = transform::create_cpu(b, n, num_threads, std::string(impl), num_regs, check_error != 0, h->ttype);
		h->g = new gint(size_t(1) << n, b);
		return h;
	}
	catch (const std::exception &e)
	{
		g_last_error = e.what();
		return nullptr;
	}
}

REF_API const char *ref_type(void *p) { return static_cast<ref_handle *>(p)->ttype.c_str(); }

REF_API void ref_destroy(void *p)
{
	ref_handle *h = static_cast<ref_handle *>(p);
	if (h == nullptr) return;
	delete h->t; delete h->g; delete h;
}

REF_API void ref_set(void *p, uint32_t a) { static_cast<ref_handle *>(p)->t->set(a); }
REF_API void ref_square_dup(void *p, int dup) { static_cast<ref_handle *>(p)->t->squareDup(dup != 0); }
REF_API void ref_square_mul(void *p, int32_t a) { static_cast<ref_handle *>(p)->t->squareMul(a); }
REF_API void ref_init_multiplicand(void *p, size_t src) { static_cast<ref_handle *>(p)->t->initMultiplicand(src); }
REF_API void ref_mul(void *p) { static_cast<ref_handle *>(p)->t->mul(); }
REF_API void ref_copy(void *p, size_t dst, size_t src) { static_cast<ref_handle *>(p)->t->copy(dst, src); }
REF_API double ref_get_error(void *p) { return static_cast<ref_handle *>(p)->t->getError(); }

/* count squareDup calls with dup flags from `bits` (one byte per squaring),
   the inner loop of genefer::prp (src/genefer.h:508-527) without GL steps. */
REF_API void ref_run_squarings(void *p, const uint8_t *bits, size_t count)
{
	transform *const t = static_cast<ref_handle *>(p)->t;
	for (size_t i = 0; i < count; ++i) t->squareDup(bits[i] != 0);
}

/* transform::getInt (src/transform.h:234-239): raw signed digits. */
REF_API void ref_get_zi(void *p, int32_t *out)
{
	ref_handle *h = static_cast<ref_handle *>(p);
	h->t->getInt(*h->g);
	std::memcpy(out, h->g->data(), (size_t(1) << h->n) * sizeof(int32_t));
}

/* transform::setInt (src/transform.h:241-246): balances, then setZi. */
REF_API void ref_set_zi(void *p, const int32_t *in)
{
	ref_handle *h = static_cast<ref_handle *>(p);
	std::memcpy(h->g->data(), in, (size_t(1) << h->n) * sizeof(int32_t));
	h->g->reset();
	h->t->setInt(*h->g);
}

/* saveContext payload of register 0 (src/transformCPUi32.h:839-846),
   written through the reference's `file` class to a temporary file. */
REF_API long ref_save_raw(void *p, void *out, size_t out_size)
{
	ref_handle *h = static_cast<ref_handle *>(p);
	char path[] = "/tmp/gfref_ctx_XXXXXX";
	const int fd = mkstemp(path);
	if (fd < 0) return -1;
	close(fd);
	{
		file f(path, "wb", false);
		h->t->saveContext(f, 1);
	}
	FILE *const fp = std::fopen(path, "rb");
	if (fp == nullptr) { std::remove(path); return -1; }
	int kind = 0;
	long got = -1;
	if (std::fread(&kind, sizeof(kind), 1, fp) == 1) got = static_cast<long>(std::fread(out, 1, out_size, fp));
	std::fclose(fp);
	std::remove(path);
	return got;
}
