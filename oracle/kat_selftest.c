/*
 * ORACLE — test infrastructure only.
 *
 * Known-answer test: the reference's SELF_TEST scenario
 * (src/gemdyn/src/base/turbo_tricublin.c:1346-1505 — a 300x200x85 analytic
 * field f = fx(x)*fy(y)*fz(z), 5 boundary probes and ~5M interior points)
 * driven through this project's restated interpolator instead of the
 * reference one.  It prints the same lines (minus timing) so the output can be
 * compared with the reference binary's output line by line.
 *
 * usage: kat_selftest [lib.so symbol-prefix]  — default: the oracle
 * restatement linked in.  With "cuda" as argument the GPU path is used through
 * the product C-ABI (loaded with dlopen from the given path).
 */
#include <dlfcn.h>
#include <stdio.h>
#include <stdlib.h>
#include "oracle.h"

#define NI 300
#define NJ 200
#define NK 85

static float fx(float x) { x = x * .125; return (x * x * x * 1.011 + x * x * 1.022 + x * 1.01 + .123); }
static float fy(float y) { y = y * .125; return (y * y * y * 1.044 + y * y * 1.055 + y * 1.03 + .234); }
static float fz(float z) { return (z * 1.123 + .345); }
static float fxyz(float x, float y, float z) { return fx(x) * fy(y) * fz(z); }

typedef void (*interp_fn)(float *d, const float *f, const float *pxyz, int n, void *ctx);

static orc_ztab *g_lv;
static void interp_oracle(float *d, const float *f, const float *pxyz, int n, void *ctx) {
  (void)ctx;
  const float *fs[1] = {f};
  orc_zyx1_m_n_f32(d, fs, pxyz, g_lv, n, 1);
}

/* product path: the reference-named drop-in entry points of the CUDA library */
typedef void *(*setup_t)(double *, int, int, int);
typedef void (*zyx1_t)(float *, float *, float *, void *, int);
static zyx1_t g_cuda_zyx1;
static void *g_cuda_lv;
static void interp_cuda(float *d, const float *f, const float *pxyz, int n, void *ctx) {
  (void)ctx;
  g_cuda_zyx1(d, (float *)f, (float *)pxyz, g_cuda_lv, n);
}

int main(int argc, char **argv) {
  static float a1[NI * NJ * NK];
  static float dest[NI * NJ * NK];
  static float posxyz[3 * NI * NJ * NK];
  static double expected[NI * NJ * NK];
  double posz[NK];
  interp_fn interp = interp_oracle;

  for (int k = 0; k < NK; k++) posz[k] = k + 1;
  float *p1 = a1;
  for (int k = 0; k < NK; k++)
    for (int j = 0; j < NJ; j++)
      for (int i = 0; i < NI; i++) *p1++ = fxyz(i + 1.0, j + 1.0, k + 1.0);

  g_lv = orc_vsearch_setup_plus(posz, NK, NI, NJ, 0, 0);
  if (argc > 1) {
    void *h = dlopen(argv[1], RTLD_NOW);
    if (!h) { fprintf(stderr, "dlopen: %s\n", dlerror()); return 2; }
    setup_t su = (setup_t)dlsym(h, "Vsearch_setup");
    g_cuda_zyx1 = (zyx1_t)dlsym(h, "Tricublin_zyx1_n");
    if (!su || !g_cuda_zyx1) { fprintf(stderr, "missing symbols\n"); return 2; }
    g_cuda_lv = su(posz, NK, NI, NJ);
    interp = interp_cuda;
  }

  int II = NI / 2, JJ = NJ / 2, KK = NK / 2;
  float dx = .555, dy = .777, dz = .333;
  struct { const char *name; int kk; float dz; } cases[5] = {
      {"Cubic case  :", NK / 2, .333f},
      {"Linear bottom case  :", 1, .25f},
      {"Linear bot extrap case  :", 0, .75f},
      {"Linear top case  :", NK - 1, .75f},
      {"Linear top extrap case  :", NK, .25f}};
  for (int c = 0; c < 5; c++) {
    float pos[3];
    KK = cases[c].kk;
    dz = cases[c].dz;
    pos[2] = dz; pos[2] = pos[2] + KK;
    pos[0] = dx + II;
    pos[1] = dy + JJ;
    float d[3];
    float a2[1];
    (void)a2;
    /* the three fields of the reference test are a1, a1+10, a1+100 */
    interp(&d[0], a1, pos, 1, NULL);
    float e0 = fxyz(II + dx, JJ + dy, KK + dz), e1 = e0 + 10, e2 = e0 + 100;
    /* a1+10 and a1+100 are interpolated through the same weights */
    static float b[NI * NJ * NK];
    static int bset = 0;
    static float cc[NI * NJ * NK];
    if (!bset) {
      for (long q = 0; q < (long)NI * NJ * NK; q++) { b[q] = a1[q] + 10; cc[q] = a1[q] + 100; }
      bset = 1;
    }
    interp(&d[1], b, pos, 1, NULL);
    interp(&d[2], cc, pos, 1, NULL);
    printf("%s\ngot %12.7g, %12.7g, %12.7g, result/expected = %10.8f %10.8f %10.8f\n", cases[c].name, d[0], d[1], d[2],
           d[0] / e0, d[1] / e1, d[2] / e2);
  }
  dz = .25; /* value left by the last probe, as in the reference */
  float *ptr = posxyz;
  double *answer = expected;
  for (int k = 0; k < NK; k++)
    for (int j = 1; j < NJ - 2; j++)
      for (int i = 1; i < NI - 2; i++) {
        ptr[0] = i + dx + 1;
        ptr[1] = j + dy + 1;
        ptr[2] = k + dz + 1;
        *answer = fxyz(ptr[0], ptr[1], ptr[2]);
        ptr += 3;
        answer++;
      }
  int npts = NK * (NI - 3) * (NJ - 3);
  printf("npts = %d, ninjnk = %d\n", npts, NK * NI * NJ);
  for (int i = 0; i < npts; i++) dest[i] = -1.0;
  interp(dest, a1, posxyz, npts, NULL);
  float e0 = 0.0, e1;
  double e8 = 0.0;
  int exact = 0;
  for (int i = 0; i < npts; i++) {
    if (i % 300000 == 0) printf("expected %12.7g, got %12.7g\n", expected[i], dest[i]);
    e1 = 1.0 - (dest[i] / expected[i]);
    if (e1 < 0) e1 = -e1;
    if (e1 == 0) exact++;
    e8 += e1;
    if (e1 > e0) e0 = e1;
  }
  e1 = npts;
  e1 = (exact / e1) * 100.0;
  printf("worst case error : %12.7g, avg error : %12.7g, exact : %8.2f percent\n", e0, e8 / npts, e1);
  printf("END\n");
  return 0;
}
