/* A C program that uses this library exactly as a C caller of SHAFFT would:
 * through include/shafft/shafft.h, the single-rank MPI shim and
 * libshafft.so, with no Python in between.  Built and run by
 * tests/test_c_caller.py.
 *
 *   shafft_c_caller cpu   configuration objects, plan state machine, layout
 *                         and axis queries, error reporting (no GPU needed)
 *   shafft_c_caller gpu   transforms with analytic answers: a plane wave
 *                         (ND, config-object initialisation), a sinusoid
 *                         (FFT1D), the buffer swap, fused normalize
 *
 * Prints one line per check and exits non-zero if any failed. */
#include <math.h>
#include <mpi.h>
#include <shafft/shafft.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static int failures = 0;

static void check(int ok, const char* what, const char* detail) {
  printf("%s %s%s%s\n", ok ? "PASS" : "FAIL", what, detail ? " : " : "", detail ? detail : "");
  if (!ok) failures++;
}

static void check_rc(int rc, int want, const char* what) {
  char last[128] = {0}, buf[200];
  shafftLastErrorMessage(last, (int)sizeof(last));
  snprintf(buf, sizeof(buf), "rc=%d want=%d last='%s'", rc, want, last);
  check(rc == want, what, rc == want ? NULL : buf);
}

static int cpu_checks(void) {
  char name[64] = {0};
  check(shafftGetBackendName() != NULL && strcmp(shafftGetBackendName(), "sm100") == 0,
        "backend name is sm100", NULL);
  int major = -1, minor = -1, patch = -1;
  shafftGetVersion(&major, &minor, &patch);
  snprintf(name, sizeof(name), "%d.%d.%d", major, minor, patch);
  check(major == 1 && minor == 1 && patch == 0, "version 1.1.0", name);

  /* configuration object: single rank resolves to commDims {1,1,1}, nda 0 */
  size_t shape[3] = {64, 64, 32};
  shafft_nd_config_t cfg;
  memset(&cfg, 0, sizeof(cfg));
  int rc = shafftConfigNDInit(&cfg, 3, shape, SHAFFT_C2C, NULL, 0, SHAFFT_MINIMIZE_NDA,
                              SHAFFT_LAYOUT_REDISTRIBUTED, 0, MPI_COMM_WORLD);
  check_rc(rc, SHAFFT_SUCCESS, "shafftConfigNDInit");
  check(cfg.allocElements == 64 * 64 * 32, "config allocElements = N", NULL);
  check(cfg.initial.localElements == 64 * 64 * 32 && cfg.nda == 0, "config initial layout", NULL);
  check(cfg.commDims && cfg.commDims[0] == 1 && cfg.commDims[1] == 1 && cfg.commDims[2] == 1,
        "config commDims resolved to 1,1,1", NULL);

  void* plan = NULL;
  check_rc(shafftNDCreate(&plan), SHAFFT_SUCCESS, "shafftNDCreate");
  check_rc(shafftNDInitFromConfig(plan, &cfg), SHAFFT_SUCCESS, "shafftNDInitFromConfig");
  int configured = 0;
  shafftIsConfigured(plan, &configured);
  check(configured == 1, "plan configured", NULL);
  size_t alloc = 0, global = 0;
  check_rc(shafftGetAllocSize(plan, &alloc), SHAFFT_SUCCESS, "shafftGetAllocSize");
  check(alloc == 64 * 64 * 32, "allocSize = N", NULL);
  shafftGetGlobalSize(plan, &global);
  check(global == 64 * 64 * 32, "globalSize = N", NULL);
  size_t sub[3] = {0}, off[3] = {9, 9, 9};
  check_rc(shafftGetLayout(plan, sub, off, SHAFFT_TENSOR_LAYOUT_CURRENT), SHAFFT_SUCCESS,
           "shafftGetLayout");
  check(sub[0] == 64 && sub[1] == 64 && sub[2] == 32 && off[0] == 0 && off[1] == 0 && off[2] == 0,
        "layout = whole tensor at offset 0", NULL);

  /* state machine and the thread-local last error */
  check_rc(shafftExecute(plan, SHAFFT_FORWARD), SHAFFT_ERR_PLAN_NOT_INIT, "execute before plan");
  check(shafftLastErrorStatus() == SHAFFT_ERR_PLAN_NOT_INIT, "last error status recorded", NULL);
  check(strcmp(shafftErrorSourceName(shafftLastErrorSource()), "SHAFFT") == 0, "error source SHAFFT",
        NULL);
  shafftClearLastError();
  check(shafftLastErrorStatus() == SHAFFT_SUCCESS, "clear last error", NULL);
  int dims2[2] = {8, 8}, grid2[2] = {1, 1};
  check_rc(shafftNDInit(plan, 2, grid2, dims2, SHAFFT_C2C, MPI_COMM_WORLD, SHAFFT_LAYOUT_REDISTRIBUTED),
           SHAFFT_ERR_INVALID_STATE, "init twice");
  check_rc(shafftNormalize(plan), SHAFFT_ERR_PLAN_NOT_INIT, "normalize before plan");
  check_rc(shafftDestroy(&plan), SHAFFT_SUCCESS, "shafftDestroy");
  check(plan == NULL, "destroy clears the handle", NULL);
  shafftConfigNDRelease(&cfg);

  /* 1-D configuration */
  size_t ln = 0, ls = 7, la = 0;
  check_rc(shafftConfiguration1D(1000, &ln, &ls, &la, SHAFFT_C2C, MPI_COMM_WORLD), SHAFFT_SUCCESS,
           "shafftConfiguration1D");
  check(ln == 1000 && ls == 0 && la == 1000, "1-D layout on one rank", NULL);
  shafft_1d_config_t c1;
  memset(&c1, 0, sizeof(c1));
  check_rc(shafftConfig1DInit(&c1, 1000, SHAFFT_Z2Z, MPI_COMM_WORLD), SHAFFT_SUCCESS,
           "shafftConfig1DInit");
  check(c1.allocElements == 1000 && c1.initial.localSize == 1000, "1-D config object", NULL);
  void* p1 = NULL;
  shafft1DCreate(&p1);
  check_rc(shafft1DInitFromConfig(p1, &c1), SHAFFT_SUCCESS, "shafft1DInitFromConfig");
  shafftDestroy(&p1);
  shafftConfig1DRelease(&c1);

  /* invalid decompositions */
  void* p2 = NULL;
  shafftNDCreate(&p2);
  int dims3[3] = {8, 8, 8}, bad[3] = {1, 1, 2};
  check(shafftNDInit(p2, 3, bad, dims3, SHAFFT_C2C, MPI_COMM_WORLD, SHAFFT_LAYOUT_REDISTRIBUTED) != 0,
        "distributed last axis refused", NULL);
  shafftDestroy(&p2);
  return 0;
}

static double cabs2(const float* v, size_t i) { return hypot((double)v[2 * i], (double)v[2 * i + 1]); }

static int gpu_checks(void) {
  /* ND: plane wave exp(+2 pi i k.x / n), k = (3, 5, 7), through a config object */
  const size_t n0 = 64, n1 = 64, n2 = 32, N = n0 * n1 * n2;
  size_t shape[3] = {n0, n1, n2};
  shafft_nd_config_t cfg;
  memset(&cfg, 0, sizeof(cfg));
  shafftConfigNDInit(&cfg, 3, shape, SHAFFT_C2C, NULL, 0, SHAFFT_MINIMIZE_NDA,
                     SHAFFT_LAYOUT_REDISTRIBUTED, 0, MPI_COMM_WORLD);
  void* plan = NULL;
  shafftNDCreate(&plan);
  check_rc(shafftNDInitFromConfig(plan, &cfg), SHAFFT_SUCCESS, "ND init from config");
  check_rc(shafftPlan(plan), SHAFFT_SUCCESS, "shafftPlan");
  void *data = NULL, *work = NULL;
  check_rc(shafftAllocBufferF(cfg.allocElements, &data), SHAFFT_SUCCESS, "shafftAllocBufferF");
  shafftAllocBufferF(cfg.allocElements, &work);
  float* host = (float*)malloc(2 * N * sizeof(float));
  const double tau = 6.283185307179586;
  for (size_t a = 0; a < n0; ++a)
    for (size_t b = 0; b < n1; ++b)
      for (size_t c = 0; c < n2; ++c) {
        const double ph = tau * (3.0 * a / n0 + 5.0 * b / n1 + 7.0 * c / n2);
        const size_t i = (a * n1 + b) * n2 + c;
        host[2 * i] = (float)cos(ph);
        host[2 * i + 1] = (float)sin(ph);
      }
  shafftCopyToBufferF(data, host, N);
  check_rc(shafftSetBuffers(plan, data, work), SHAFFT_SUCCESS, "shafftSetBuffers");
  check_rc(shafftExecute(plan, SHAFFT_FORWARD), SHAFFT_SUCCESS, "execute forward");
  void *d2 = NULL, *w2 = NULL;
  shafftGetBuffers(plan, &d2, &w2);
  check(d2 == work && w2 == data, "result reported in the other buffer (swap)", NULL);
  shafftCopyFromBufferF(host, d2, N);
  const size_t peak = (3 * n1 + 5) * n2 + 7;
  double rest = 0;
  for (size_t i = 0; i < N; ++i)
    if (i != peak) rest = fmax(rest, cabs2(host, i));
  char msg[128];
  snprintf(msg, sizeof(msg), "|X[k]| = %.3f (want %zu), max elsewhere %.2e", cabs2(host, peak), N, rest);
  check(fabs(cabs2(host, peak) - (double)N) < 1e-5 * N && rest < 1e-5 * N, "plane wave spectrum", msg);

  /* normalize, backward, normalize: the plane wave again */
  check_rc(shafftNormalize(plan), SHAFFT_SUCCESS, "normalize");
  check_rc(shafftExecuteNormalized(plan, SHAFFT_BACKWARD), SHAFFT_SUCCESS, "execute normalized backward");
  shafftGetBuffers(plan, &d2, &w2);
  shafftCopyFromBufferF(host, d2, N);
  double err = 0;
  for (size_t a = 0; a < n0; ++a)
    for (size_t b = 0; b < n1; ++b)
      for (size_t c = 0; c < n2; ++c) {
        const double ph = tau * (3.0 * a / n0 + 5.0 * b / n1 + 7.0 * c / n2);
        const size_t i = (a * n1 + b) * n2 + c;
        err = fmax(err, hypot(host[2 * i] - cos(ph), host[2 * i + 1] - sin(ph)));
      }
  snprintf(msg, sizeof(msg), "max error %.2e", err);
  check(err < 1e-5, "round trip restores the input", msg);
  shafftFreeBufferF(data);
  shafftFreeBufferF(work);
  shafftDestroy(&plan);
  shafftConfigNDRelease(&cfg);

  /* FFT1D: sinusoid cos(2 pi 17 j / n) -> peaks n/2 at 17 and n-17 */
  const size_t n = 4096;
  size_t ln = 0, ls = 0, la = 0;
  shafftConfiguration1D(n, &ln, &ls, &la, SHAFFT_C2C, MPI_COMM_WORLD);
  void* p1 = NULL;
  shafft1DCreate(&p1);
  check_rc(shafft1DInit(p1, n, ln, ls, SHAFFT_C2C, MPI_COMM_WORLD), SHAFFT_SUCCESS, "shafft1DInit");
  check_rc(shafftPlan(p1), SHAFFT_SUCCESS, "FFT1D plan");
  shafftAllocBufferF(la, &data);
  shafftAllocBufferF(la, &work);
  for (size_t j = 0; j < n; ++j) {
    host[2 * j] = (float)cos(tau * 17.0 * j / n);
    host[2 * j + 1] = 0.f;
  }
  shafftCopyToBufferF(data, host, n);
  shafftSetBuffers(p1, data, work);
  check_rc(shafftExecute(p1, SHAFFT_FORWARD), SHAFFT_SUCCESS, "FFT1D forward");
  shafftGetBuffers(p1, &d2, &w2);
  shafftCopyFromBufferF(host, d2, n);
  rest = 0;
  for (size_t k = 0; k < n; ++k)
    if (k != 17 && k != n - 17) rest = fmax(rest, cabs2(host, k));
  snprintf(msg, sizeof(msg), "|X[17]| = %.3f |X[n-17]| = %.3f max elsewhere %.2e", cabs2(host, 17),
           cabs2(host, n - 17), rest);
  check(fabs(cabs2(host, 17) - n / 2.0) < 1e-5 * n && fabs(cabs2(host, n - 17) - n / 2.0) < 1e-5 * n &&
            rest < 1e-5 * n,
        "FFT1D sinusoid spectrum", msg);
  shafftFreeBufferF(data);
  shafftFreeBufferF(work);
  shafftDestroy(&p1);
  free(host);
  return 0;
}

int main(int argc, char** argv) {
  MPI_Init(&argc, &argv);
  const char* mode = argc > 1 ? argv[1] : "cpu";
  if (strcmp(mode, "gpu") == 0)
    gpu_checks();
  else
    cpu_checks();
  shafftFinalize();
  MPI_Finalize();
  printf("%d failure(s)\n", failures);
  return failures ? 1 : 0;
}
