/*
 * C restatement of upstream s2fft's Price-McEwen latitudinal steps (float64).
 *
 * TEST INFRASTRUCTURE ONLY: the timed CPU baseline of bench.py and a checker in
 * tests/. The product library never links or loads it.
 *
 * Follows, operation by operation, the numpy functions that the oracle package
 * restates in Python (oracle/recursion.py):
 *   s2o_precompute   <- s2fft/recursions/price_mcewen.py:118-255 (generate_precomputes_jax:
 *                       lrenorm seeds, vsign, cpi, cp2; NaN/inf mapped to 0 as at 251-253)
 *   s2o_inverse_lat  <- s2fft/transforms/otf_recursions.py:15-171 (inverse_latitudinal_step)
 *   s2o_forward_lat  <- s2fft/transforms/otf_recursions.py:432-588 (forward_latitudinal_step)
 * The m-recursion renormalises in log space at every step (exp and log per term),
 * NaN terms are dropped from the sums (np.nansum), exactly as upstream. Two
 * liberties, neither of which changes a result beyond summation order: the terms of
 * degrees not yet reached by the recursion (upstream multiplies them by an exact zero)
 * are skipped, and the rings are split over OpenMP threads (every ring's recursion is
 * independent; the forward sums the threads' partial coefficients at the end).
 *
 * Layouts (row-major, complex = interleaved double pairs):
 *   flm [L][2L-1], ftm [nth][ncol] (ncol = 2L for mwss/healpix, 2L-1 otherwise),
 *   lrenorm [2][nth][n], vsign [2L-1][n], cpi, cp2 [L+1][n], n = L - L0.
 */
#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

static double nz(double x) { return isfinite(x) ? x : 0.0; }

/* price_mcewen.py:118-255 (through the oracle's restatement, oracle/recursion.py). */
void s2o_precompute(int L, int spin, int nth, const double* beta, int L0, double* lrenorm,
                    double* vsign, double* cpi, double* cp2) {
  const int mm = -spin;
  const int n = L - L0;
  const int R = L + 1;
  /* cpi / cp2 columns before the roll, then rolled per column by L - l - 1 */
  double* a = (double*)malloc(sizeof(double) * R);
  double* b = (double*)malloc(sizeof(double) * R);
  for (int k = 0; k < n; ++k) {
    const double el = (double)(L0 + k);
    for (int r = 0; r < R; ++r) a[r] = b[r] = 0.0;
    a[0] = 2.0 / sqrt(2.0 * el);
    for (int m = 2; m <= L; ++m) {
      a[m - 1] = 2.0 / sqrt((double)m * (2.0 * el + 1.0 - (double)m));
      b[m - 1] = a[m - 1] / a[m - 2];
    }
    const int sh = L - (L0 + k) - 1;
    for (int r = 0; r < R; ++r) {
      const int src = ((r - sh) % R + R) % R;
      cpi[(size_t)r * n + k] = nz(a[src]);
      cp2[(size_t)r * n + k] = nz(b[src]);
    }
  }
  free(a);
  free(b);
  /* sign table (206-210) */
  for (int j = 0; j < 2 * L - 1; ++j) {
    double ms = j < L - 1 ? ((j % 2) ? -1.0 : 1.0) : 1.0;
    if (j < L - 1) ms *= (abs(mm + 1 + L) % 2) ? -1.0 : 1.0;
    for (int k = 0; k < n; ++k) {
      const double ls = (abs(mm + L0 + k) % 2) ? -1.0 : 1.0;
      vsign[(size_t)j * n + k] = ms * ls;
    }
  }
  /* log-seeds (212-243): row = 2 l log|cos(b/2)|, then row += log((2l+2-i)/(i-1))/2 +
   * log|tan(-b/2)| for i = 2 .. L+|mm|+1; half h takes the row at i = l -+ mm + 1 */
  const int imax = L + abs(mm) + 1;
#pragma omp parallel for schedule(dynamic, 4)
  for (int t = 0; t < nth; ++t) {
    const double lt = log(fabs(tan(-beta[t] / 2.0)));
    const double lc2 = log(fabs(cos(beta[t] / 2.0)));
    for (int k = 0; k < n; ++k) {
      const int el = L0 + k;
      const int h0 = el + mm + 1, h1 = el - mm + 1;
      double row = lc2 * (2.0 * el);
      double v0 = 0.0, v1 = 0.0;
      if (h0 == 1) v0 = row;
      if (h1 == 1) v1 = row;
      const int last = h0 > h1 ? h0 : h1;
      for (int i = 2; i <= imax && i <= last; ++i) {
        row = row + log((2.0 * el + 2.0 - i) / (double)(i - 1)) / 2.0 + lt;
        if (h0 == i) v0 = row;
        if (h1 == i) v1 = row;
      }
      lrenorm[((size_t)0 * nth + t) * n + k] = nz(v0);
      lrenorm[((size_t)1 * nth + t) * n + k] = nz(v1);
    }
  }
}

/* column index helper: python-style negative indices */
static inline int wrap(int c, int ncols) { return c < 0 ? c + ncols : c; }

typedef struct {
  int L, L0, n, nth, spin, mo_first, reality;
  const double* beta;
  const double* lrenorm;
  const double* vsign;
  const double* cpi;
  const double* cp2;
} Lat;

/* One ring's recursion over both halves (otf_recursions.py:85-171 / 500-588). For every
 * (column, active degree k) the macro TERM(col, ftm column, k, weight) receives
 * weight = d * vsign * exp(lrenorm). */
#define RING_LOOP(TERM)                                                                    \
  do {                                                                                     \
    const int L = P->L, L0 = P->L0, n = P->n;                                              \
    const int mm = -P->spin;                                                               \
    const double c = cos(P->beta[t]), s = sin(P->beta[t]);                                 \
    const double omc = 1.0 - c;                                                            \
    for (int i = 0; i < 2; ++i) {                                                          \
      if (P->reality && i == 0) continue;                                                  \
      const int mo = (P->mo_first && i == 0) ? 1 : 0;                                      \
      const int lind = L - 1 - L0;                                                         \
      const int sind = i == 0 ? 0 : -1;                                                    \
      const int sgn = i == 0 ? 1 : -1;                                                     \
      const double* lr0 = P->lrenorm + ((size_t)i * P->nth + t) * n;                       \
      for (int k = 0; k < n; ++k) {                                                        \
        d0[k] = 1.0;                                                                       \
        d1[k] = 1.0;                                                                       \
        lr[k] = lr0[k];                                                                    \
        en[k] = 0.0;                                                                       \
      }                                                                                    \
      {                                                                                    \
        const double el = (double)(L0 + lind);                                             \
        const double half = i == 0 ? el + mm + 1 : el - mm + 1;                            \
        const double lam = (omc * (el + 1.0) + c * ((double)(2 - L) + el) - half) / s;     \
        d1[lind] = P->cpi[lind] * d0[lind] * lam;                                          \
      }                                                                                    \
      {                                                                                    \
        const int col = sind;                                                              \
        const int k = lind;                                                                \
        const double w = d0[k] * P->vsign[(size_t)wrap(col, 2 * L - 1) * n + k] * exp(lr[k]); \
        TERM(col, col + mo, k, w);                                                         \
      }                                                                                    \
      for (int k = (lind - 1 < 0 ? 0 : lind - 1); k <= lind; ++k) {                        \
        const int col = sind + sgn;                                                        \
        const double w = d1[k] * P->vsign[(size_t)wrap(col, 2 * L - 1) * n + k] * exp(lr[k]); \
        TERM(col, col + mo, k, w);                                                         \
      }                                                                                    \
      const int last = L - 1 + i;                                                          \
      for (int m = 2; m < last; ++m) {                                                     \
        const int kact = L - m - 1 - L0 < 0 ? 0 : L - m - 1 - L0;                          \
        const double* cpm = P->cpi + (size_t)(m - 1) * n;                                  \
        const double* cqm = P->cp2 + (size_t)(m - 1) * n;                                  \
        const double colb = (double)(m - L + 1);                                           \
        for (int k = kact; k < n; ++k) {                                                   \
          const double el = (double)(L0 + k);                                              \
          const double half = i == 0 ? el + mm + 1 : el - mm + 1;                          \
          const double lam = (omc * (el + 1.0) + c * (colb + el) - half) / s;              \
          en[k] = cpm[k] * d1[k] * lam - cqm[k] * d0[k];                                   \
        }                                                                                  \
        if (L - m - 1 - L0 >= 0) en[L - m - 1 - L0] = 1.0;                                 \
        const int col = sind + sgn * m;                                                    \
        const double* vs = P->vsign + (size_t)wrap(col, 2 * L - 1) * n;                    \
        for (int k = kact; k < n; ++k) {                                                   \
          const double w = en[k] * vs[k] * exp(lr[k]);                                     \
          TERM(col, col + mo, k, w);                                                       \
        }                                                                                  \
        for (int k = kact; k < n; ++k) {                                                   \
          const double mag = fabs(en[k]);                                                  \
          const double nd0 = d1[k] / mag;                                                  \
          d1[k] = en[k] / mag;                                                             \
          d0[k] = nd0;                                                                     \
          lr[k] = lr[k] + log(mag);                                                        \
        }                                                                                  \
      }                                                                                    \
    }                                                                                      \
  } while (0)

/* otf_recursions.py:15-171. flm: the normalised coefficients [L][2L-1] (complex);
 * ftm out [nth][ncol] (complex), zeroed here. mo_first = 1 for mwss / healpix. */
void s2o_inverse_lat(int L, int spin, int L0, int reality, int mo_first, int nth,
                     const double* beta, const double* lrenorm, const double* vsign,
                     const double* cpi, const double* cp2, const double* flm, int ncol,
                     double* ftm, int nthreads) {
  Lat Q = {L, L0, L - L0, nth, spin, mo_first, reality, beta, lrenorm, vsign, cpi, cp2};
  const Lat* P = &Q;
  const int W = 2 * L - 1;
  const int n = L - L0;
  /* flm transposed to [column][k] so that a column's degrees are contiguous */
  double* ft = (double*)malloc(sizeof(double) * 2 * (size_t)W * n);
  for (int col = 0; col < W; ++col)
    for (int k = 0; k < n; ++k) {
      ft[((size_t)col * n + k) * 2] = flm[((size_t)(L0 + k) * W + col) * 2];
      ft[((size_t)col * n + k) * 2 + 1] = flm[((size_t)(L0 + k) * W + col) * 2 + 1];
    }
  memset(ftm, 0, sizeof(double) * 2 * (size_t)nth * ncol);
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel
  {
    double* d0 = (double*)malloc(sizeof(double) * n);
    double* d1 = (double*)malloc(sizeof(double) * n);
    double* lr = (double*)malloc(sizeof(double) * n);
    double* en = (double*)malloc(sizeof(double) * n);
#pragma omp for schedule(dynamic, 1)
    for (int t = 0; t < nth; ++t) {
      double* row = ftm + (size_t)t * ncol * 2;
#define INV_TERM(col, fcol, k, w)                                                    \
  do {                                                                               \
    double* o_ = row + 2 * wrap(fcol, ncol);                                         \
    const double* fv_ = ft + ((size_t)wrap(col, W) * n + (k)) * 2;                   \
    const double tr_ = (w) * fv_[0], ti_ = (w) * fv_[1];                             \
    if (!isnan(tr_)) o_[0] += tr_;                                                   \
    if (!isnan(ti_)) o_[1] += ti_;                                                   \
  } while (0)
      RING_LOOP(INV_TERM);
#undef INV_TERM
    }
    free(d0);
    free(d1);
    free(lr);
    free(en);
  }
  free(ft);
}

/* otf_recursions.py:432-588. ftm [nth][ncol] (complex, weights applied); flm out
 * [L][2L-1] (complex), zeroed here. */
void s2o_forward_lat(int L, int spin, int L0, int reality, int mo_first, int nth,
                     const double* beta, const double* lrenorm, const double* vsign,
                     const double* cpi, const double* cp2, const double* ftm, int ncol,
                     double* flm, int nthreads) {
  Lat Q = {L, L0, L - L0, nth, spin, mo_first, reality, beta, lrenorm, vsign, cpi, cp2};
  const Lat* P = &Q;
  const int W = 2 * L - 1;
  const int n = L - L0;
  if (nthreads > 0) omp_set_num_threads(nthreads);
  const int T = omp_get_max_threads();
  /* per thread partial sums [column][k] (complex) */
  double* part = (double*)calloc((size_t)T * W * n * 2, sizeof(double));
#pragma omp parallel
  {
    double* d0 = (double*)malloc(sizeof(double) * n);
    double* d1 = (double*)malloc(sizeof(double) * n);
    double* lr = (double*)malloc(sizeof(double) * n);
    double* en = (double*)malloc(sizeof(double) * n);
    double* acc = part + (size_t)omp_get_thread_num() * W * n * 2;
#pragma omp for schedule(dynamic, 1)
    for (int t = 0; t < nth; ++t) {
      const double* row = ftm + (size_t)t * ncol * 2;
#define FWD_TERM(col, fcol, k, w)                                                    \
  do {                                                                               \
    const double* gv_ = row + 2 * wrap(fcol, ncol);                                  \
    double* a_ = acc + ((size_t)wrap(col, W) * n + (k)) * 2;                         \
    const double tr_ = (w) * gv_[0], ti_ = (w) * gv_[1];                             \
    if (!isnan(tr_)) a_[0] += tr_;                                                   \
    if (!isnan(ti_)) a_[1] += ti_;                                                   \
  } while (0)
      RING_LOOP(FWD_TERM);
#undef FWD_TERM
    }
    free(d0);
    free(d1);
    free(lr);
    free(en);
  }
  memset(flm, 0, sizeof(double) * 2 * (size_t)L * W);
  for (int th = 0; th < T; ++th) {
    const double* a = part + (size_t)th * W * n * 2;
    for (int col = 0; col < W; ++col)
      for (int k = 0; k < n; ++k) {
        flm[((size_t)(L0 + k) * W + col) * 2] += a[((size_t)col * n + k) * 2];
        flm[((size_t)(L0 + k) * W + col) * 2 + 1] += a[((size_t)col * n + k) * 2 + 1];
      }
  }
  free(part);
}

int s2o_max_threads(void) { return omp_get_max_threads(); }
