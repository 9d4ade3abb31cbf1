/* exact.c - ORACLE (test infrastructure only): exact enumeration of small Ising models.
 *
 * Restates drift/solvers/exact.py:20-49 (enumerate all 2^n configurations, take the minimum and
 * keep the whole spectrum) as a Gray-code walk: consecutive configurations differ in one spin, so
 * the energy is updated with the local field in O(n) per step instead of an O(n^2) einsum, and
 * n up to 30 fits in memory (the reference caps at 24, exact.py:25-26). The spin of bit b is
 * 1 - 2b (bit 0 -> +1), the convention of exact.py:21-23.
 *
 * Besides the ground energy it returns Boltzmann averages at a list of inverse temperatures
 * (correctness part (b) of the engine: marginals and observables against exact enumeration):
 * <E>, <E^2>, <|m|>, <m^2> and the single-site magnetisations <s_i>.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct ExactOut {
  double e_min;
  uint64_t argmin;     /* first configuration index (natural order) reaching e_min */
  double* mean_e;      /* [n_beta] */
  double* mean_e2;     /* [n_beta] */
  double* mean_absm;   /* [n_beta] */
  double* mean_m2;     /* [n_beta] */
  double* site_mag;    /* [n_beta][n] or NULL */
  double* spectrum;    /* [2^n] energies in natural index order, or NULL */
} ExactOut;

static inline int ctz64(uint64_t x) { return __builtin_ctzll(x); }

/* J dense row-major [n][n] (symmetric, zero diagonal), h [n]. */
int oracle_exact(int n, const double* J, const double* h, int n_beta, const double* betas, ExactOut* out) {
  if (n < 1 || n > 30) return 1;
  const uint64_t N = 1ULL << n;
  double* f = (double*)malloc(sizeof(double) * n); /* f_i = sum_j J_ij s_j */
  int8_t* s = (int8_t*)malloc((size_t)n);
  /* pass 1: minimum (and spectrum) */
  for (int i = 0; i < n; ++i) s[i] = 1;
  double E = 0.0;
  for (int i = 0; i < n; ++i) {
    double fi = 0.0;
    for (int j = 0; j < n; ++j) fi += J[(size_t)i * n + j];
    f[i] = fi;
  }
  for (int i = 0; i < n; ++i) E += -0.5 * f[i] - h[i];
  uint64_t idx = 0;  /* natural index of the current configuration */
  double emin = E;
  uint64_t arg = 0;
  if (out->spectrum) out->spectrum[0] = E;
  for (uint64_t k = 1; k < N; ++k) {
    int i = ctz64(k);
    double dE = 2.0 * s[i] * (f[i] + h[i]);
    E += dE;
    for (int j = 0; j < n; ++j) f[j] -= 2.0 * J[(size_t)j * n + i] * s[i];
    s[i] = (int8_t)-s[i];
    idx ^= 1ULL << i;
    if (out->spectrum) out->spectrum[idx] = E;
    if (E < emin || (E == emin && idx < arg)) {
      emin = E;
      arg = idx;
    }
  }
  out->e_min = emin;
  out->argmin = arg;
  if (n_beta > 0) {
    /* pass 2: Boltzmann weights exp(-beta (E - e_min)) */
    double* Z = (double*)calloc((size_t)n_beta, sizeof(double));
    for (int b = 0; b < n_beta; ++b) {
      out->mean_e[b] = out->mean_e2[b] = out->mean_absm[b] = out->mean_m2[b] = 0.0;
      if (out->site_mag)
        for (int i = 0; i < n; ++i) out->site_mag[(size_t)b * n + i] = 0.0;
    }
    for (int i = 0; i < n; ++i) s[i] = 1;
    for (int i = 0; i < n; ++i) {
      double fi = 0.0;
      for (int j = 0; j < n; ++j) fi += J[(size_t)i * n + j];
      f[i] = fi;
    }
    E = 0.0;
    for (int i = 0; i < n; ++i) E += -0.5 * f[i] - h[i];
    int msum = n;
    for (uint64_t k = 0; k < N; ++k) {
      if (k > 0) {
        int i = ctz64(k);
        E += 2.0 * s[i] * (f[i] + h[i]);
        for (int j = 0; j < n; ++j) f[j] -= 2.0 * J[(size_t)j * n + i] * s[i];
        msum -= 2 * s[i];
        s[i] = (int8_t)-s[i];
      }
      const double m = (double)msum / n;
      for (int b = 0; b < n_beta; ++b) {
        const double w = exp(-betas[b] * (E - emin));
        Z[b] += w;
        out->mean_e[b] += w * E;
        out->mean_e2[b] += w * E * E;
        out->mean_absm[b] += w * fabs(m);
        out->mean_m2[b] += w * m * m;
        if (out->site_mag)
          for (int i = 0; i < n; ++i) out->site_mag[(size_t)b * n + i] += w * s[i];
      }
    }
    for (int b = 0; b < n_beta; ++b) {
      out->mean_e[b] /= Z[b];
      out->mean_e2[b] /= Z[b];
      out->mean_absm[b] /= Z[b];
      out->mean_m2[b] /= Z[b];
      if (out->site_mag)
        for (int i = 0; i < n; ++i) out->site_mag[(size_t)b * n + i] /= Z[b];
    }
    free(Z);
  }
  free(f);
  free(s);
  return 0;
}
