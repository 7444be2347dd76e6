// gf_gint.cpp -- host-side residue utilities of genefer's `gint`
// (src/gint.h:40-225): canonical digits, res64/old64 and the Gerbicz-Li
// hash.  They run once per test or per check on N host digits, as in the
// reference, and are exported through the same C ABI as the engine.
#include <cstddef>
#include <cstdint>

#define GFC_API extern "C" __attribute__((visibility("default")))

namespace {

// One carry sweep with digit rule `canon` (true: [0, b); false: (-b/2, b/2]).
inline int64_t sweep(int32_t *d, size_t size, int32_t base, int64_t f, bool canon, bool stop_at_zero)
{
	for (size_t i = 0; i < size; ++i)
	{
		f += d[i];
		int32_t r = static_cast<int32_t>(f % base);
		if (canon) { if (r < 0) r += base; }
		else { if (r > base / 2) r -= base; if (r <= -base / 2) r += base; }
		d[i] = r;
		f -= r;
		f /= base;
		if (stop_at_zero && (f == 0)) break;
	}
	return f;
}

inline uint64_t rotl64(uint64_t x, unsigned n) { return (x << n) | (x >> ((64 - n) & 63)); }

}  // namespace

// gint::unbalance (src/gint.h:40-102): digits in [0, b); -1 stays as d[0] = -1.
GFC_API void gfc_gint_unbalance(int32_t *d, size_t size, uint32_t b)
{
	const int32_t base = static_cast<int32_t>(b);
	int64_t f = sweep(d, size, base, 0, true, false);
	while (f != 0)
	{
		f = sweep(d, size, base, -f, true, true);   // f x^size = -f
		if (f == 1)
		{
			bool zero = true;
			for (size_t i = 0; i < size; ++i) if (d[i] != 0) { zero = false; break; }
			if (zero) { d[0] = -1; break; }
		}
	}
}

// gint::balance (src/gint.h:104-149): digits in (-b/2, b/2].
GFC_API void gfc_gint_balance(int32_t *d, size_t size, uint32_t b)
{
	const int32_t base = static_cast<int32_t>(b);
	int64_t f = sweep(d, size, base, 0, false, false);
	while (f != 0) f = sweep(d, size, base, -f, false, true);
}

// gint::isOne (src/gint.h:169-202) on canonical digits.
GFC_API int gfc_gint_is_one(const int32_t *d, size_t size, uint32_t b, uint64_t *res64, uint64_t *old64)
{
	bool one = (d[0] == 1);
	for (size_t i = 1; one && (i < size); ++i) one = (d[i] == 0);
	uint64_t r = 0, w = 1;
	for (size_t i = 0; i < size; ++i) { r += static_cast<uint64_t>(static_cast<uint32_t>(d[i])) * w; w *= b; }
	uint64_t o = 0;
	for (size_t i = 8; i != 0; --i) o = (o << 8) | static_cast<uint8_t>(d[size - i]);
	if (res64 != nullptr) *res64 = r;
	if (old64 != nullptr) *old64 = o;
	return one ? 1 : 0;
}

// gint::gethash64 (src/gint.h:204-219) on canonical digits.
GFC_API uint64_t gfc_gint_hash64(const int32_t *d, size_t size)
{
	uint64_t h = 0;
	for (size_t i = 0; i < size; ++i)
	{
		const uint32_t a = static_cast<uint32_t>(d[i]);
		h += a;
		h ^= rotl64(a + 0xc39d8a0552b073e8ull, static_cast<unsigned>((17 * static_cast<uint64_t>(a) + 5) % 64));
	}
	return h;
}
