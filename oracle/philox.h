/*
 * Counter-based Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random
 * numbers: as easy as 1, 2, 3", SC'11) and the seeded matrix draws used by
 * the tests and the benchmark.  Test infrastructure: the product library has
 * its own device generator, checked bit-for-bit against this one.
 *
 * Stream layout: key = (seed, matrix_id), counter = (idx_lo, idx_hi, 0, 0)
 * where idx is the element's column-major linear index.
 *
 * Draws:
 *   uniform f32   : ((w0 >> 8) * 2^-23) - 1                     in [-1, 1)
 *   uniform f64   : ((w0:w1 >> 11) * 2^-52) - 1                 in [-1, 1)
 *   wide          : sign(w2) * (1 + frac) * 2^e, frac from w0(:w1),
 *                   e = (w3 % 21) - 10                          |x| in [2^-10, 2^11)
 *   diag f32/f64  : 1 + (uniform + 1) / 2                       in [1, 2)
 */
#ifndef MUBLIS_ORACLE_PHILOX_H
#define MUBLIS_ORACLE_PHILOX_H

#include <math.h>
#include <stdint.h>

typedef struct { uint32_t v[4]; } philox4x32_t;

static inline philox4x32_t philox4x32_10_ctr(const uint32_t ctr[4], const uint32_t key[2]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int round = 0; round < 10; ++round) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
    uint32_t n1 = (uint32_t)p1;
    uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    uint32_t n3 = (uint32_t)p0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  philox4x32_t r = {{c0, c1, c2, c3}};
  return r;
}

static inline philox4x32_t philox4x32_10(uint64_t index, uint32_t seed, uint32_t matrix_id) {
  const uint32_t ctr[4] = {(uint32_t)index, (uint32_t)(index >> 32), 0u, 0u};
  const uint32_t key[2] = {seed, matrix_id};
  return philox4x32_10_ctr(ctr, key);
}

enum { PHILOX_DRAW_UNIFORM = 0, PHILOX_DRAW_WIDE = 1, PHILOX_DRAW_DIAG = 2 };

static inline float philox_draw_f32(uint64_t index, uint32_t seed, uint32_t matrix_id, int kind) {
  philox4x32_t r = philox4x32_10(index, seed, matrix_id);
  float u = (float)(r.v[0] >> 8) * 0x1p-23f - 1.0f;
  if (kind == PHILOX_DRAW_DIAG) return 1.0f + (u + 1.0f) * 0.5f;
  if (kind == PHILOX_DRAW_WIDE) {
    float mant = 1.0f + (float)(r.v[0] >> 9) * 0x1p-23f;
    int e = (int)(r.v[3] % 21u) - 10;
    float x = ldexpf(mant, e);
    return (r.v[2] & 1u) ? -x : x;
  }
  return u;
}

static inline double philox_draw_f64(uint64_t index, uint32_t seed, uint32_t matrix_id, int kind) {
  philox4x32_t r = philox4x32_10(index, seed, matrix_id);
  uint64_t bits = (((uint64_t)r.v[0] << 32) | r.v[1]) >> 11;
  double u = (double)bits * 0x1p-52 - 1.0;
  if (kind == PHILOX_DRAW_DIAG) return 1.0 + (u + 1.0) * 0.5;
  if (kind == PHILOX_DRAW_WIDE) {
    double mant = 1.0 + (double)(bits >> 1) * 0x1p-52;
    int e = (int)(r.v[3] % 21u) - 10;
    double x = ldexp(mant, e);
    return (r.v[2] & 1u) ? -x : x;
  }
  return u;
}

#endif
