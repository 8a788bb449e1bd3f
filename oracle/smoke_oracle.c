/*
 * CPU oracle for the smoke-simulation step: a plain-C restatement of the
 * reference's Numba kernels (LCEBurton/python-game-engine, src/cfd/backends/numba)
 * plus the project's own FP64 restatement of the convergent multigrid pieces.
 *
 * TEST INFRASTRUCTURE ONLY. It is the parity checker for the CUDA library and
 * the CPU baseline timed beside it; the product never links or calls it.
 * Build: oracle/Makefile (gcc -O2 -fopenmp -ffp-contract=off).
 */
#include <math.h>
#include <stdint.h>

/* SplitMix64 finaliser (Steele, Lea, Flood 2014): the counter-based hash behind
 * the plume source's seeded velocity noise. The CUDA library uses the same
 * function so that both sides draw identical noise without copying arrays. */
static inline unsigned long long sg_mix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

/* Uniform noise in [-amp, amp) keyed by (seed, step, component, row, column). */
double sg_noise(unsigned long long seed, long step, int comp, long j, long i, double amp) {
  unsigned long long h = sg_mix64(seed ^ sg_mix64((unsigned long long)step));
  h = sg_mix64(h ^ (((unsigned long long)comp << 62) | ((unsigned long long)j << 31) |
                    (unsigned long long)i));
  double u = (double)(h >> 11) * (1.0 / 9007199254740992.0);
  return amp * (2.0 * u - 1.0);
}

#define REAL float
#define SFX _f32
#include "smoke_oracle_impl.h"
#undef REAL
#undef SFX

#define REAL double
#define SFX _f64
#include "smoke_oracle_impl.h"
#undef REAL
#undef SFX
