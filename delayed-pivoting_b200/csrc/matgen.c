/*
 * Seeded synthetic inputs for the delayed-pivoting LU (host, no CUDA).
 *
 * The reference publishes no dataset; its workloads are N(0,1) matrices from a
 * seeded mt19937_64 with planted tiny (x1e-18) and exact-zero columns.  This
 * file produces those bytes reproducibly on any host so the CUDA library,
 * the CPU reference and the oracle all see the same input.
 *
 *   generator  MT19937-64 (Matsumoto & Nishimura 2004), the engine of C++
 *              std::mt19937_64; column j of a matrix is filled from its own
 *              engine seeded with splitmix64(seed + j * 0x9E3779B97F4A7C15),
 *              so columns can be generated in parallel.
 *   uniform    (x >> 11) * 2^-53 in [0, 1)
 *   normal     Marsaglia's polar method, both outputs used in order.
 *   columns    planted columns are a seeded Fisher-Yates shuffle of 0..n-1:
 *              the first n_tiny are scaled by tiny_scale, the next n_zero are
 *              set to exact zero.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

#define NN 312
#define MM 156
#define MATRIX_A 0xB5026F5AA96619E9ULL
#define UM 0xFFFFFFFF80000000ULL
#define LM 0x7FFFFFFFULL

typedef struct {
  uint64_t mt[NN];
  int mti;
} mt64;

static void mt64_seed(mt64 *s, uint64_t seed) {
  s->mt[0] = seed;
  for (int i = 1; i < NN; ++i)
    s->mt[i] = 6364136223846793005ULL * (s->mt[i - 1] ^ (s->mt[i - 1] >> 62)) + (uint64_t)i;
  s->mti = NN;
}

static uint64_t mt64_next(mt64 *s) {
  if (s->mti >= NN) {
    int i;
    for (i = 0; i < NN - MM; ++i) {
      uint64_t x = (s->mt[i] & UM) | (s->mt[i + 1] & LM);
      s->mt[i] = s->mt[i + MM] ^ (x >> 1) ^ ((x & 1ULL) ? MATRIX_A : 0ULL);
    }
    for (; i < NN - 1; ++i) {
      uint64_t x = (s->mt[i] & UM) | (s->mt[i + 1] & LM);
      s->mt[i] = s->mt[i + (MM - NN)] ^ (x >> 1) ^ ((x & 1ULL) ? MATRIX_A : 0ULL);
    }
    uint64_t x = (s->mt[NN - 1] & UM) | (s->mt[0] & LM);
    s->mt[NN - 1] = s->mt[MM - 1] ^ (x >> 1) ^ ((x & 1ULL) ? MATRIX_A : 0ULL);
    s->mti = 0;
  }
  uint64_t x = s->mt[s->mti++];
  x ^= (x >> 29) & 0x5555555555555555ULL;
  x ^= (x << 17) & 0x71D67FFFEDA60000ULL;
  x ^= (x << 37) & 0xFFF7EEE000000000ULL;
  x ^= (x >> 43);
  return x;
}

static uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}

static double mt64_uniform(mt64 *s) { return (double)(mt64_next(s) >> 11) * (1.0 / 9007199254740992.0); }

/* Returns the count-th output (1-based) of an engine seeded with `seed`, for
 * checking the engine against std::mt19937_64 (seed 5489: 10000th output is
 * 9981545732273789042 by the C++ standard). */
uint64_t dpgen_mt64_nth(uint64_t seed, int count) {
  mt64 s;
  mt64_seed(&s, seed);
  uint64_t v = 0;
  for (int i = 0; i < count; ++i) v = mt64_next(&s);
  return v;
}

static void fill_normal(mt64 *s, double *x, long long len) {
  long long i = 0;
  while (i < len) {
    double u, v, q;
    do {
      u = 2.0 * mt64_uniform(s) - 1.0;
      v = 2.0 * mt64_uniform(s) - 1.0;
      q = u * u + v * v;
    } while (q >= 1.0 || q == 0.0);
    const double f = sqrt(-2.0 * log(q) / q);
    x[i++] = u * f;
    if (i < len) x[i++] = v * f;
  }
}

/* a(0:m, 0:n) ~ N(0,1), column-major with leading dimension lda. */
void dpgen_normal_matrix(int m, int n, double *a, long long lda, uint64_t seed) {
#pragma omp parallel for schedule(static)
  for (int j = 0; j < n; ++j) {
    mt64 s;
    mt64_seed(&s, splitmix64(seed + (uint64_t)j * 0x9E3779B97F4A7C15ULL));
    fill_normal(&s, a + (size_t)j * (size_t)lda, m);
  }
}

/* Vector of `len` N(0,1) values from engine splitmix64(seed). */
void dpgen_normal_vector(double *x, long long len, uint64_t seed) {
  mt64 s;
  mt64_seed(&s, splitmix64(seed));
  fill_normal(&s, x, len);
}

/* Seeded Fisher-Yates over 0..n-1; first n_tiny columns scaled by
 * tiny_scale, next n_zero set to 0.  The chosen indices are written to
 * tiny_cols / zero_cols (either may be NULL). */
int dpgen_plant_columns(int m, int n, double *a, long long lda, uint64_t seed, int n_tiny,
                        double tiny_scale, int n_zero, int *tiny_cols, int *zero_cols) {
  if (n_tiny < 0 || n_zero < 0 || n_tiny + n_zero > n) return -1;
  int *perm = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  if (!perm) return -1;
  for (int j = 0; j < n; ++j) perm[j] = j;
  mt64 s;
  mt64_seed(&s, splitmix64(seed ^ 0xD1B54A32D192ED03ULL));
  for (int i = n - 1; i > 0; --i) {
    const uint64_t r = mt64_next(&s);
    const int j = (int)(((unsigned __int128)r * (unsigned __int128)(i + 1)) >> 64);
    const int t = perm[i];
    perm[i] = perm[j];
    perm[j] = t;
  }
  for (int t = 0; t < n_tiny; ++t) {
    double *c = a + (size_t)perm[t] * (size_t)lda;
    for (int i = 0; i < m; ++i) c[i] *= tiny_scale;
    if (tiny_cols) tiny_cols[t] = perm[t];
  }
  for (int t = 0; t < n_zero; ++t) {
    double *c = a + (size_t)perm[n_tiny + t] * (size_t)lda;
    for (int i = 0; i < m; ++i) c[i] = 0.0;
    if (zero_cols) zero_cols[t] = perm[n_tiny + t];
  }
  free(perm);
  return 0;
}

/* Uniform integer in [lo, hi] and uniform double in [0,1) streams for the
 * batched / served workload generators: out[i] for i < count. */
void dpgen_uniform(double *out, long long count, uint64_t seed) {
  mt64 s;
  mt64_seed(&s, splitmix64(seed ^ 0x2545F4914F6CDD1DULL));
  for (long long i = 0; i < count; ++i) out[i] = mt64_uniform(&s);
}
