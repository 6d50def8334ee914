// ORACLE — test infrastructure only. Nothing in the product links, imports or
// runs this code; tests/, the smoke check and bench.py's CPU-baseline leg use
// it as the checker.
//
// JavaScript numeric helpers shared by the two CPU restatements:
//   - js_toint32: ECMAScript ToInt32 (what `^`, `|`, `&` apply to a Number)
//   - js_hash: Solver._hash, src/solver.js:162-164
//       ((xi*92837111) ^ (yi*689287499) ^ (zi*283923481)) >>> 0) & (T-1)
//     with each product formed in double precision, as JavaScript does.
//   - js_cell: Math.floor(p * (1 / cellSize)), src/solver.js:166-172
#pragma once
#include <cmath>
#include <cstdint>

namespace oracle {

// ECMAScript 2023 §7.1.6 ToInt32.
inline int32_t js_toint32(double x) {
  if (!std::isfinite(x)) return 0;
  double t = std::trunc(x);
  double m = std::fmod(t, 4294967296.0);  // exact
  if (m < 0) m += 4294967296.0;
  if (m >= 2147483648.0) m -= 4294967296.0;
  return (int32_t)m;
}

// Math.floor(p * inv) with p a float32 typed-array element (exact in double).
inline double js_cell(double p, double inv) { return std::floor(p * inv); }

inline uint32_t js_hash(double xi, double yi, double zi, uint32_t table_size) {
  int32_t a = js_toint32(xi * 92837111.0);
  int32_t b = js_toint32(yi * 689287499.0);
  int32_t c = js_toint32(zi * 283923481.0);
  uint32_t h = (uint32_t)(a ^ b ^ c);   // `>>> 0`
  return h & (table_size - 1u);         // `& (tableSize - 1)`
}

// Math.max(0, x) keeps NaN, unlike std::max.
inline double js_max0(double x) { return (x != x) ? x : (x > 0.0 ? x : 0.0); }
// Math.sign(q) || 1
inline double js_sign_or1(double q) { return q > 0 ? 1.0 : (q < 0 ? -1.0 : 1.0); }

}  // namespace oracle
