/* Project-written FP64 mixed-radix FFT exposing the FFTW subset used by the
 * reference (test infrastructure only; see fftw3.h in this folder).
 *
 * Algorithm: recursive decimation in time. A line of length n = p*m (p the
 * smallest prime factor) is split into p interleaved sub-sequences of length
 * m, each transformed recursively, then recombined with twiddles
 * w_n^{r k} and a direct length-p DFT. Cost O(n * sum of prime factors),
 * i.e. O(n log n) for the 2,3,5,7-smooth sizes the reference uses
 * (code/forcefield0.c:219-245 rounds the top grid to such sizes).
 * Twiddle angles use (r*k mod n) for accuracy.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "fftw3.h"

struct msm_shim_plan {
  int n[3];
  fftw_complex *a;
  int sign;
};

static int smallest_factor(int n) {
  if (n % 2 == 0) return 2;
  for (int f = 3; (long)f * f <= n; f += 2)
    if (n % f == 0) return f;
  return n;
}

/* out[k] = sum_j in[j*stride] * exp(sign * 2 pi i j k / n), k < n */
static void fft_rec(const fftw_complex *in, long stride, fftw_complex *out,
                    int n, int sign, fftw_complex *tmp) {
  if (n == 1) {
    out[0] = in[0];
    return;
  }
  const double twopi = 6.283185307179586476925286766559;
  int p = smallest_factor(n);
  int m = n / p;
  for (int r = 0; r < p; r++)
    fft_rec(in + r * stride, stride * p, out + (long)r * m, m, sign, tmp);
  for (int k = 0; k < m; k++) {
    for (int r = 0; r < p; r++) {
      long e = ((long)r * k) % n;
      double ang = sign * twopi * (double)e / (double)n;
      tmp[r] = out[(long)r * m + k] * (cos(ang) + I * sin(ang));
    }
    for (int s = 0; s < p; s++) {
      fftw_complex acc = 0;
      for (int r = 0; r < p; r++) {
        long e = ((long)r * s) % p;
        double ang = sign * twopi * (double)e / (double)p;
        acc += tmp[r] * (cos(ang) + I * sin(ang));
      }
      out[k + (long)s * m] = acc;
    }
  }
}

static void fft_line(fftw_complex *a, int n, long stride, int sign,
                     fftw_complex *line, fftw_complex *res,
                     fftw_complex *tmp) {
  for (int j = 0; j < n; j++) line[j] = a[j * stride];
  fft_rec(line, 1, res, n, sign, tmp);
  for (int j = 0; j < n; j++) a[j * stride] = res[j];
}

void msm_shim_fft3d(fftw_complex *a, int n0, int n1, int n2, int sign) {
  int nmax = n0 > n1 ? n0 : n1;
  nmax = nmax > n2 ? nmax : n2;
  fftw_complex *buf = malloc(sizeof(fftw_complex) * 3 * (size_t)nmax);
  fftw_complex *line = buf, *res = buf + nmax, *tmp = buf + 2 * nmax;
  for (int i = 0; i < n0; i++)
    for (int j = 0; j < n1; j++)
      fft_line(a + ((long)i * n1 + j) * n2, n2, 1, sign, line, res, tmp);
  for (int i = 0; i < n0; i++)
    for (int k = 0; k < n2; k++)
      fft_line(a + (long)i * n1 * n2 + k, n1, n2, sign, line, res, tmp);
  for (int j = 0; j < n1; j++)
    for (int k = 0; k < n2; k++)
      fft_line(a + (long)j * n2 + k, n0, (long)n1 * n2, sign, line, res, tmp);
  free(buf);
}

fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in,
                           fftw_complex *out, int sign, unsigned flags) {
  (void)out; /* the reference only plans in-place transforms */
  (void)flags;
  fftw_plan p = malloc(sizeof *p);
  p->n[0] = n0;
  p->n[1] = n1;
  p->n[2] = n2;
  p->a = in;
  p->sign = sign;
  return p;
}

void fftw_execute(const fftw_plan p) {
  msm_shim_fft3d(p->a, p->n[0], p->n[1], p->n[2], p->sign);
}

void fftw_destroy_plan(fftw_plan p) { free(p); }
void *fftw_malloc(unsigned long n) { return malloc(n); }
void fftw_free(void *p) { free(p); }
