/*
 * oracle_fft_body.h -- type-generic body of the CPU oracle (test
 * infrastructure only).  Included twice by oracle_fft.c with REAL bound to
 * double and to long double.  See oracle_fft.c for what is restated.
 */
#define OCAT2(a, b) a##b
#define OCAT(a, b) OCAT2(a, b)
#define FN(name) OCAT(name, SUFFIX)

typedef struct {
  REAL re, im;
} FN(cplx);
#define CPLX FN(cplx)

/* Exact twiddle: exp(sign * 2*pi*i * m / n) with m reduced modulo n first. */
static CPLX FN(twiddle)(int64_t m, int64_t n, int sign) {
  m %= n;
  if (m < 0) m += n;
  /* use symmetry so that the angle stays in [0, pi/4] where cos/sin are
   * best conditioned */
  int64_t m8 = 8 * m;
  CPLX w;
  REAL ang;
  if (m8 <= n) {
    ang = 2 * PI_R * (REAL)m / (REAL)n;
    w.re = COS(ang);
    w.im = SIN(ang);
  } else if (m8 <= 3 * n) {
    ang = 2 * PI_R * (REAL)(n - 4 * m) / (REAL)(4 * n); /* pi/2 - theta */
    w.re = SIN(ang);
    w.im = COS(ang);
  } else if (m8 <= 5 * n) {
    ang = 2 * PI_R * (REAL)(2 * m - n) / (REAL)(2 * n); /* theta - pi */
    w.re = -COS(ang);
    w.im = -SIN(ang);
  } else if (m8 <= 7 * n) {
    ang = 2 * PI_R * (REAL)(3 * n - 4 * m) / (REAL)(4 * n); /* 3pi/2 - theta */
    w.re = -SIN(ang);
    w.im = -COS(ang);
  } else {
    ang = 2 * PI_R * (REAL)(n - m) / (REAL)n; /* 2pi - theta */
    w.re = COS(ang);
    w.im = -SIN(ang);
  }
  if (sign < 0) w.im = -w.im;
  return w;
}

/* A 1-D plan: factors, twiddle table w_n^m (m < n) or a Bluestein sub-plan. */
typedef struct FN(plan1d) {
  int64_t n;
  int sign;
  int nf;
  int64_t f[ORACLE_MAX_FACTORS];
  CPLX* tw;  /* n entries, w_n^m for the direct mixed-radix path */
  /* Bluestein */
  int blue;
  int64_t m;              /* power-of-two convolution length */
  CPLX* chirp;            /* n entries: exp(sign*i*pi*k^2/n) */
  CPLX* hspec;            /* m entries: FFT_m of the conjugate chirp kernel */
  struct FN(plan1d)* sub; /* forward length-m plan */
  struct FN(plan1d)* subi; /* backward length-m plan */
} FN(plan1d);

static void FN(plan_free)(FN(plan1d) * p) {
  if (!p) return;
  free(p->tw);
  free(p->chirp);
  free(p->hspec);
  FN(plan_free)(p->sub);
  FN(plan_free)(p->subi);
  free(p);
}

static int FN(smallest_factor)(int64_t n) {
  if (n % 4 == 0) return 4;
  if (n % 2 == 0) return 2;
  for (int64_t p = 3; p * p <= n; p += 2)
    if (n % p == 0) return (int)p;
  return n > ORACLE_DIRECT_PRIME_MAX ? -1 : (int)n;
}

/* largest prime factor of n */
static int64_t FN(largest_prime)(int64_t n) {
  int64_t best = 1;
  for (int64_t p = 2; p * p <= n; ++p)
    while (n % p == 0) {
      best = p;
      n /= p;
    }
  if (n > 1) best = n > best ? n : best;
  return best;
}

static void FN(exec1d)(const FN(plan1d) * p, CPLX* x, CPLX* y, CPLX* scratch);

static FN(plan1d) * FN(plan_make)(int64_t n, int sign) {
  FN(plan1d)* p = (FN(plan1d)*)calloc(1, sizeof(FN(plan1d)));
  if (!p) return NULL;
  p->n = n;
  p->sign = sign;
  if (n > 1 && FN(largest_prime)(n) > ORACLE_DIRECT_PRIME_MAX) {
    /* Bluestein */
    p->blue = 1;
    int64_t m = 1;
    while (m < 2 * n - 1) m <<= 1;
    p->m = m;
    p->chirp = (CPLX*)malloc(sizeof(CPLX) * (size_t)n);
    p->hspec = (CPLX*)calloc((size_t)m, sizeof(CPLX));
    p->sub = FN(plan_make)(m, -1);
    p->subi = FN(plan_make)(m, +1);
    if (!p->chirp || !p->hspec || !p->sub || !p->subi) {
      FN(plan_free)(p);
      return NULL;
    }
    for (int64_t k = 0; k < n; ++k) {
      /* k^2 mod 2n in exact integer arithmetic (unsigned 128-bit product) */
      unsigned __int128 kk = (unsigned __int128)k * (unsigned __int128)k;
      int64_t r = (int64_t)(kk % (unsigned __int128)(2 * n));
      /* exp(sign*i*pi*r/n) = w_{2n}^{r} with the given sign */
      p->chirp[k] = FN(twiddle)(r, 2 * n, sign);
    }
    /* kernel h[j] = conj(chirp[|j|]) laid out cyclically */
    CPLX* h = (CPLX*)calloc((size_t)m, sizeof(CPLX));
    CPLX* t = (CPLX*)malloc(sizeof(CPLX) * (size_t)m);
    CPLX* s = (CPLX*)malloc(sizeof(CPLX) * (size_t)m);
    if (!h || !t || !s) {
      free(h);
      free(t);
      free(s);
      FN(plan_free)(p);
      return NULL;
    }
    for (int64_t k = 0; k < n; ++k) {
      h[k].re = p->chirp[k].re;
      h[k].im = -p->chirp[k].im;
      if (k) h[m - k] = h[k];
    }
    FN(exec1d)(p->sub, h, p->hspec, s);
    free(h);
    free(t);
    free(s);
    return p;
  }
  int64_t r = n;
  while (r > 1) {
    int f = FN(smallest_factor)(r);
    if (f < 0 || p->nf >= ORACLE_MAX_FACTORS) {
      FN(plan_free)(p);
      return NULL;
    }
    p->f[p->nf++] = f;
    r /= f;
  }
  p->tw = (CPLX*)malloc(sizeof(CPLX) * (size_t)n);
  if (!p->tw) {
    FN(plan_free)(p);
    return NULL;
  }
  for (int64_t m = 0; m < n; ++m) p->tw[m] = FN(twiddle)(m, n, sign);
  return p;
}

/* Stockham mixed-radix DIT; x is read, y receives the result, scratch has n
 * entries.  x may equal y.  */
static void FN(stockham)(const FN(plan1d) * p, const CPLX* x, CPLX* y, CPLX* scratch) {
  const int64_t n = p->n;
  if (n == 1) {
    y[0] = x[0];
    return;
  }
  /* ping-pong between two buffers; choose the start so the last stage lands
   * in y */
  CPLX* bufs[2];
  int cur;
  {
    CPLX* a = scratch;
    CPLX* b = y;
    /* after nf stages the data sits in bufs[(start + nf) & 1]; want y */
    if (p->nf & 1) {
      bufs[0] = a;
      bufs[1] = b;
    } else {
      bufs[0] = b;
      bufs[1] = a;
    }
    cur = 0;
    if (bufs[0] != x) memmove(bufs[0], x, sizeof(CPLX) * (size_t)n);
  }
  CPLX v[ORACLE_DIRECT_PRIME_MAX + 4];
  int64_t l = 1;
  for (int st = 0; st < p->nf; ++st) {
    const int64_t rad = p->f[st];
    const int64_t lp = l * rad;
    const int64_t ns = n / lp; /* number of output subsequences s' */
    const CPLX* A = bufs[cur];
    CPLX* B = bufs[cur ^ 1];
    const int64_t twstep = n / lp; /* w_{l'}^{e} = w_n^{e * n/l'} */
    const int64_t pstep = n / rad; /* w_p^{e} = w_n^{e * n/p} */
    CPLX wp[ORACLE_DIRECT_PRIME_MAX + 4]; /* w_p^e, e < rad */
    for (int64_t e = 0; e < rad; ++e) wp[e] = p->tw[e * pstep];
    for (int64_t s = 0; s < ns; ++s) {
      for (int64_t k = 0; k < l; ++k) {
        for (int64_t r = 0; r < rad; ++r) {
          CPLX a = A[(s + ns * r) * l + k];
          CPLX w = p->tw[r * k * twstep]; /* r*k*twstep < rad*l*(n/lp) = n */
          v[r].re = a.re * w.re - a.im * w.im;
          v[r].im = a.re * w.im + a.im * w.re;
        }
        for (int64_t q = 0; q < rad; ++q) {
          REAL sr = 0, si = 0;
          int64_t e = 0; /* (r*q) mod rad, advanced by q per r */
          for (int64_t r = 0; r < rad; ++r) {
            CPLX w = wp[e];
            sr += v[r].re * w.re - v[r].im * w.im;
            si += v[r].re * w.im + v[r].im * w.re;
            e += q;
            if (e >= rad) e -= rad;
          }
          B[s * lp + k + l * q].re = sr;
          B[s * lp + k + l * q].im = si;
        }
      }
    }
    cur ^= 1;
    l = lp;
  }
}

/* scratch must hold max(n, 3*m) entries for a Bluestein plan (m = conv
 * length), n entries otherwise. */
static void FN(exec1d)(const FN(plan1d) * p, CPLX* x, CPLX* y, CPLX* scratch) {
  if (!p->blue) {
    FN(stockham)(p, x, y, scratch);
    return;
  }
  const int64_t n = p->n, m = p->m;
  CPLX* a = scratch;
  CPLX* b = scratch + m;
  CPLX* s = scratch + 2 * m;
  for (int64_t k = 0; k < m; ++k) {
    if (k < n) {
      CPLX c = p->chirp[k];
      a[k].re = x[k].re * c.re - x[k].im * c.im;
      a[k].im = x[k].re * c.im + x[k].im * c.re;
    } else {
      a[k].re = 0;
      a[k].im = 0;
    }
  }
  FN(stockham)(p->sub, a, b, s);
  for (int64_t k = 0; k < m; ++k) {
    CPLX h = p->hspec[k];
    REAL re = b[k].re * h.re - b[k].im * h.im;
    REAL im = b[k].re * h.im + b[k].im * h.re;
    b[k].re = re;
    b[k].im = im;
  }
  FN(stockham)(p->subi, b, a, s);
  const REAL inv = (REAL)1 / (REAL)m;
  for (int64_t k = 0; k < n; ++k) {
    CPLX c = p->chirp[k];
    REAL re = (a[k].re * c.re - a[k].im * c.im) * inv;
    REAL im = (a[k].re * c.im + a[k].im * c.re) * inv;
    y[k].re = re;
    y[k].im = im;
  }
}

static int64_t FN(scratch_len)(const FN(plan1d) * p) {
  return p->blue ? 3 * p->m + p->n : 2 * p->n;
}

/* Transform one axis of a row-major tensor held in work (long double or
 * double complex), in place.  Lines of a strided axis are gathered in groups
 * of neighbouring lines (consecutive inner indices) that fill one 64-byte
 * cache line, so each gathered cache line is used whole; every line is
 * transformed on its own, exactly as when taken one at a time. */
#ifndef ORACLE_LINE_GROUP
#define ORACLE_LINE_GROUP ((int64_t)(64 / sizeof(CPLX)) > 1 ? (int64_t)(64 / sizeof(CPLX)) : 1)
#endif
static int FN(axis_pass)(CPLX* data, int ndim, const int64_t* dims, int axis, int sign,
                         int nthreads) {
  const int64_t n = dims[axis];
  if (n == 1) return 0;
  int64_t inner = 1, outer = 1;
  for (int a = axis + 1; a < ndim; ++a) inner *= dims[a];
  for (int a = 0; a < axis; ++a) outer *= dims[a];
  FN(plan1d)* p = FN(plan_make)(n, sign);
  if (!p) return -2;
  const int64_t G = inner >= ORACLE_LINE_GROUP ? ORACLE_LINE_GROUP : 1;
  /* row pitch of the gathered lines: one element more than a power-of-two
   * length, so that the G rows do not alias onto the same cache sets */
  const int64_t ld = G > 1 ? n + 1 : n;
  const int64_t per_outer = (inner + G - 1) / G;
  const int64_t groups = outer * per_outer;
  const int64_t slen = FN(scratch_len)(p);
  int err = 0;
#ifdef _OPENMP
  int nt = nthreads > 0 ? nthreads : omp_get_max_threads();
#pragma omp parallel num_threads(nt)
#endif
  {
    CPLX* lines = (CPLX*)malloc(sizeof(CPLX) * (size_t)(G * ld + slen));
    if (!lines) {
#ifdef _OPENMP
#pragma omp atomic write
#endif
      err = -2;
    } else {
      CPLX* scr = lines + G * ld;
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
      for (int64_t gi = 0; gi < groups; ++gi) {
        const int64_t o = gi / per_outer, i0 = (gi % per_outer) * G;
        const int64_t g = inner - i0 < G ? inner - i0 : G;
        CPLX* base = data + o * n * inner + i0;
        for (int64_t k = 0; k < n; ++k)
          for (int64_t j = 0; j < g; ++j) lines[j * ld + k] = base[k * inner + j];
        for (int64_t j = 0; j < g; ++j) FN(exec1d)(p, lines + j * ld, lines + j * ld, scr);
        for (int64_t k = 0; k < n; ++k)
          for (int64_t j = 0; j < g; ++j) base[k * inner + j] = lines[j * ld + k];
      }
      free(lines);
    }
  }
  FN(plan_free)(p);
  return err;
}

static int FN(fftaxes)(const double* in, double* out, int ndim, const int64_t* dims,
                       int naxes, const int* axes, int sign, int nthreads) {
  int64_t total = 1;
  for (int a = 0; a < ndim; ++a) total *= dims[a];
  CPLX* w = (CPLX*)malloc(sizeof(CPLX) * (size_t)total);
  if (!w) return -2;
#ifdef _OPENMP
  const int nt = nthreads > 0 ? nthreads : omp_get_max_threads();
#pragma omp parallel for schedule(static) num_threads(nt)
#endif
  for (int64_t i = 0; i < total; ++i) {
    w[i].re = (REAL)in[2 * i];
    w[i].im = (REAL)in[2 * i + 1];
  }
  int rc = 0;
  for (int i = 0; i < naxes && rc == 0; ++i)
    rc = FN(axis_pass)(w, ndim, dims, axes[i], sign, nthreads);
  if (rc == 0) {
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(nt)
#endif
    for (int64_t i = 0; i < total; ++i) {
      out[2 * i] = (double)w[i].re;
      out[2 * i + 1] = (double)w[i].im;
    }
  }
  free(w);
  return rc;
}

static int FN(fftnd)(const double* in, double* out, int ndim, const int64_t* dims, int sign,
                     int nthreads) {
  int axes[64];
  if (ndim > 64) return -1;
  /* fastest axis first, like the reference's subplan ordering */
  for (int a = 0; a < ndim; ++a) axes[a] = ndim - 1 - a;
  return FN(fftaxes)(in, out, ndim, dims, ndim, axes, sign, nthreads);
}

/* naive separable DFT: per axis, X[k] = sum_j x[j] w_n^{jk} with the exponent
 * j*k reduced modulo n in integers. */
static int FN(naive)(const double* in, double* out, int ndim, const int64_t* dims, int sign) {
  int64_t total = 1;
  for (int a = 0; a < ndim; ++a) total *= dims[a];
  CPLX* w = (CPLX*)malloc(sizeof(CPLX) * (size_t)total);
  if (!w) return -2;
  for (int64_t i = 0; i < total; ++i) {
    w[i].re = (REAL)in[2 * i];
    w[i].im = (REAL)in[2 * i + 1];
  }
  for (int axis = 0; axis < ndim; ++axis) {
    const int64_t n = dims[axis];
    int64_t inner = 1, outer = 1;
    for (int a = axis + 1; a < ndim; ++a) inner *= dims[a];
    for (int a = 0; a < axis; ++a) outer *= dims[a];
    CPLX* line = (CPLX*)malloc(sizeof(CPLX) * (size_t)n);
    if (!line) {
      free(w);
      return -2;
    }
    for (int64_t o = 0; o < outer; ++o)
      for (int64_t i = 0; i < inner; ++i) {
        CPLX* base = w + o * n * inner + i;
        for (int64_t k = 0; k < n; ++k) line[k] = base[k * inner];
        for (int64_t k = 0; k < n; ++k) {
          REAL sr = 0, si = 0;
          for (int64_t j = 0; j < n; ++j) {
            CPLX t = FN(twiddle)((j * k) % n, n, sign);
            sr += line[j].re * t.re - line[j].im * t.im;
            si += line[j].re * t.im + line[j].im * t.re;
          }
          base[k * inner].re = sr;
          base[k * inner].im = si;
        }
      }
    free(line);
  }
  for (int64_t i = 0; i < total; ++i) {
    out[2 * i] = (double)w[i].re;
    out[2 * i + 1] = (double)w[i].im;
  }
  free(w);
  return 0;
}

#undef CPLX
#undef FN
#undef OCAT
#undef OCAT2
