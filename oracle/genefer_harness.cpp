/*
 * genefer_harness.cpp -- runs genefer's OWN proof, server and check modes
 * (class genefer, src/genefer.h:1376-1600, with prp/GL/PL/server/check at
 * :479-1099) on the reference's i32 CPU transform, to produce fixtures that
 * pin the product's restatement of those modes (genefer22_b200/proof.py).
 * Test infrastructure only; built by oracle/Makefile into
 * oracle/_ref/genefer_harness from the reference sources where they lie.
 *
 *   genefer_harness <dir> <b> <n> <depth> <seed_time>
 *
 * In <dir> it writes genefer's g.proof (Proof mode) and g.cert (Server mode),
 * then runs Check mode on that certificate; genefer appends each mode's
 * result line (res64, old64, pkey, ckey) to <dir>/results.txt.
 *
 * genefer's server draws its three random exponents from std::rand after
 * std::srand(std::time(nullptr)) (src/genefer.h:844-845).  This executable
 * defines time() itself, so that the seed is <seed_time> and the certificate
 * is reproducible, and prints the three values that seed gives, computed as
 * genefer's rand32 does (src/genefer.h:768), as "rnd r1 r2 r3".
 */
#include <cstdio>
#include <cstdlib>
#include <ctime>
#include <string>
#include <unistd.h>

#include "genefer.h"

static time_t g_fixed_time = 1;

// Replaces the C library's time() for this executable (the reference code is
// compiled into it), so that genefer's server seeds std::rand with a known value.
extern "C" time_t time(time_t *t) noexcept
{
	if (t != nullptr) *t = g_fixed_time;
	return g_fixed_time;
}

static uint32_t rand32(const uint32_t rmin, const uint32_t rmax) { return (static_cast<uint32_t>(std::rand()) % (rmax - rmin)) + rmin; }

int main(int argc, char **argv)
{
	if (argc != 6)
	{
		std::fprintf(stderr, "usage: %s <dir> <b> <n> <depth> <seed_time>\n", argv[0]);
		return 2;
	}
	if (chdir(argv[1]) != 0) { std::perror("chdir"); return 2; }
	const uint32_t b = static_cast<uint32_t>(std::strtoul(argv[2], nullptr, 10));
	const uint32_t n = static_cast<uint32_t>(std::strtoul(argv[3], nullptr, 10));
	const int depth = std::atoi(argv[4]);
	g_fixed_time = static_cast<time_t>(std::strtoll(argv[5], nullptr, 10));

	genefer &g = genefer::getInstance();
	g.setFilename("g");
	if (g.check(b, n, genefer::EMode::Proof, 0, 1, "i32", depth) != genefer::EReturn::Success) return 1;
	if (g.check(b, n, genefer::EMode::Server, 0, 1, "i32", depth) != genefer::EReturn::Success) return 1;
	if (g.check(b, n, genefer::EMode::Check, 0, 1, "i32", depth) != genefer::EReturn::Success) return 1;

	std::srand(static_cast<unsigned int>(g_fixed_time)); std::rand();
	const uint32_t r1 = rand32(2, 64), r2 = rand32(16, 256), r3 = rand32(4, 65536);
	std::printf("rnd %u %u %u\n", r1, r2, r3);
	return 0;
}
