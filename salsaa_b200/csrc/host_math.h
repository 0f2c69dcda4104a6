// host_math.h — host-side modular arithmetic for table construction and the
// scalar entry points of the HEXL-compatible tier.
#pragma once
#include <cstdint>

namespace salsaa {
namespace host {

typedef unsigned __int128 u128;

inline uint64_t mulmod(uint64_t a, uint64_t b, uint64_t q) { return (uint64_t)(((u128)a * b) % q); }
inline uint64_t addmod(uint64_t a, uint64_t b, uint64_t q) { return (uint64_t)(((u128)(a % q) + (b % q)) % q); }
inline uint64_t submod(uint64_t a, uint64_t b, uint64_t q) {
  a %= q;
  b %= q;
  return a >= b ? a - b : a + (q - b);
}
inline uint64_t powmod(uint64_t a, uint64_t e, uint64_t q) {
  uint64_t r = 1 % q, b = a % q;
  while (e) {
    if (e & 1) r = mulmod(r, b, q);
    b = mulmod(b, b, q);
    e >>= 1;
  }
  return r;
}
// Extended Euclid; 0 when a has no inverse mod q.
inline uint64_t invmod(uint64_t a, uint64_t q) {
  __int128 t = 0, nt = 1, r = q, nr = a % q;
  while (nr != 0) {
    __int128 qt = r / nr, tmp = t - qt * nt;
    t = nt;
    nt = tmp;
    tmp = r - qt * nr;
    r = nr;
    nr = tmp;
  }
  if (r != 1) return 0;
  if (t < 0) t += q;
  return (uint64_t)t;
}
// Smallest primitive `order`-th root of unity (order a power of two): the
// root HEXL's NTT(n, q) uses for order 2n.  0 if none exists.
inline uint64_t minimal_root(uint64_t order, uint64_t q) {
  if (order < 2 || (order & (order - 1)) || (q - 1) % order) return 0;
  uint64_t g = 0;
  for (uint64_t x = 2; x < q && x < 100000; x++) {
    uint64_t c = powmod(x, (q - 1) / order, q);
    if (powmod(c, order / 2, q) == q - 1) {
      g = c;
      break;
    }
  }
  if (!g) return 0;
  uint64_t g2 = mulmod(g, g, q), cur = g, best = g;
  for (uint64_t i = 0; i < order / 2; i++) {
    if (cur < best) best = cur;
    cur = mulmod(cur, g2, q);
  }
  return best;
}
inline uint32_t bitrev(uint64_t x, unsigned bits) {
  uint64_t r = 0;
  for (unsigned i = 0; i < bits; i++) r |= ((x >> i) & 1) << (bits - 1 - i);
  return (uint32_t)r;
}
inline unsigned ilog2(uint64_t x) { return x ? 63u - (unsigned)__builtin_clzll(x) : 0u; }

}  // namespace host
}  // namespace salsaa
