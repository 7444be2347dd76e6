// kat_transformCUDA.cpp -- drives genefer's `transform` interface on
// transformCUDA (include/transformCUDA.h) the way genefer::quick does
// (prp + Gerbicz-Li validation, src/genefer.h:479-615, :736-748), using
// genefer's own `transform`, `gint` and `file` classes from its headers.
// Prints "b n res64 isPrp glOk ctxOk" for each (b, n) pair on the command line.
// Built by __graft_entry__.build() when the genefer sources are available.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <unistd.h>

#include <gmp.h>

#include "transform.h"
#include "transformCUDA.h"

static int ilog2(size_t x) { int r = -1; while (x != 0) { x >>= 1; ++r; } return r; }

// genefer::B_GerbiczLi (src/genefer.h:467-471)
static int B_GerbiczLi(const size_t esize)
{
	const size_t L = size_t(2) << (ilog2(esize) / 2);
	return static_cast<int>((esize - 1) / L) + 1;
}

// Context round trip through genefer's file class (src/file.h).
static bool context_roundtrip(transform *T, const uint32_t b, const uint32_t n)
{
	char path[] = "/tmp/kat_ctx_XXXXXX";
	const int fd = mkstemp(path);
	if (fd < 0) return false;
	close(fd);
	gint g0(size_t(1) << n, b), g1(size_t(1) << n, b);
	T->getInt(g0);
	{ file f(path, "wb", true); T->saveContext(f, 3); }
	T->squareDup(true);
	bool ok;
	// the kind word is this backend's own, not an EKind value such as the OpenCL
	// build's NTT3 (7); a file that carries NTT3 there is refused
	int kind = 0;
	if (FILE *fp = std::fopen(path, "rb")) { ok = (std::fread(&kind, sizeof(kind), 1, fp) == 1); std::fclose(fp); }
	else ok = false;
	ok = ok && (kind == static_cast<int>(GFC_CONTEXT_KIND));
	if (ok) { file f(path); ok = T->readContext(f, 3); }
	if (ok)
	{
		const int ntt3 = 7;
		if (FILE *fp = std::fopen(path, "r+b")) { ok = (std::fwrite(&ntt3, sizeof(ntt3), 1, fp) == 1); std::fclose(fp); }
		else ok = false;
		if (ok) { file f(path); ok = !T->readContext(f, 3); }
	}
	std::remove(path);
	T->getInt(g1);
	for (size_t i = 0; ok && (i < (size_t(1) << n)); ++i) ok = (g0.data()[i] == g1.data()[i]);
	return ok;
}

int main(int argc, char **argv)
{
	for (int a = 1; a + 1 < argc; a += 2)
	{
		const uint32_t b = static_cast<uint32_t>(std::strtoul(argv[a], nullptr, 10));
		const uint32_t n = static_cast<uint32_t>(std::strtoul(argv[a + 1], nullptr, 10));
		mpz_t E; mpz_init(E);
		mpz_ui_pow_ui(E, b, 1ul << n);
		const size_t esize = mpz_sizeinbase(E, 2);
		const int B = B_GerbiczLi(esize);

		transformCUDA tc(b, n, 0, 3);
		transform *const T = &tc;
		gint gi(size_t(1) << n, b);

		// prp (src/genefer.h:492-547)
		T->set(1);
		T->copy(1, 0);
		for (int i = static_cast<int>(esize) - 1; i >= 0; --i)
		{
			T->squareDup(mpz_tstbit(E, mp_bitcnt_t(i)) != 0);
			if ((i % B == 0) && (i / B != 0)) { T->copy(2, 0); T->mul(1); T->copy(1, 0); T->copy(0, 2); }
		}
		T->getInt(gi);
		uint64_t res64 = 0, old64 = 0;
		const bool isPrp = gi.isOne(res64, old64);

		// GL (src/genefer.h:557-615)
		T->mul(1);
		T->copy(2, 0);
		T->copy(0, 1);
		for (int i = B - 1; i >= 0; --i) T->squareDup(false);
		T->copy(1, 0);
		mpz_t res, e, t; mpz_init_set_ui(res, 0); mpz_init_set(e, E); mpz_init(t);
		while (mpz_sgn(e) != 0)
		{
			mpz_mod_2exp(t, e, static_cast<unsigned long>(B));
			mpz_add(res, res, t);
			mpz_div_2exp(e, e, static_cast<unsigned long>(B));
		}
		T->set(1);
		for (int i = static_cast<int>(mpz_sizeinbase(res, 2)) - 1; i >= 0; --i) T->squareDup(mpz_tstbit(res, mp_bitcnt_t(i)) != 0);
		T->mul(1);
		T->getInt(gi);
		const uint64_t h1 = gi.gethash64();
		T->copy(0, 2);
		T->getInt(gi);
		const uint64_t h2 = gi.gethash64();
		const bool ctx = context_roundtrip(T, b, n);
		std::printf("%u %u %016llX %d %d %d\n", b, n, static_cast<unsigned long long>(res64), isPrp ? 1 : 0, (h1 == h2) ? 1 : 0,
					ctx ? 1 : 0);
		std::fflush(stdout);
		mpz_clear(E); mpz_clear(res); mpz_clear(e); mpz_clear(t);
	}
	return 0;
}
