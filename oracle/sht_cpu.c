/*
 * sht_cpu.c -- C restatement of SpeedyTransforms' CPU transform, FP32.
 *
 * TEST INFRASTRUCTURE ONLY (the CPU baseline and a second checker): only tests/,
 * the cpu_baseline leg of bench.py and bench.py --impl reference load it; the
 * product never links it.
 *
 * Follows the reference's CPU algorithm:
 *   - Legendre synthesis, SpeedyTransforms/src/legendre.jl:2-101: per ring j, per
 *     order m <= mmax_truncation[j], per layer k, the even/odd dot products over l
 *     accumulated with fused multiply-adds in increasing l, north = even + odd,
 *     south = even - odd, optional 1/coslat;
 *   - Legendre analysis, legendre.jl:104-195: per ring j, per m, even/odd =
 *     dOmega_j (f_N +- f_S), outer-product accumulation into the coefficients;
 *   - Fourier stages, SpeedyTransforms/src/fourier.jl:129-292: unnormalised real
 *     FFT per ring and hemisphere with FFTW's r2c / c2r conventions. FFTW is not
 *     available here; a mixed-radix complex FFT (own code) transforms the northern
 *     and southern ring of a pair as one complex sequence.
 *   - Tables as SpectralTransform (spectral_transform.jl:138-172): Gaussian
 *     latitudes/weights and Legendre polynomials in FP64, stored in FP32 as the
 *     reference stores them in NF = Float32.
 * Threads (pthreads, dynamic scheduling): rings for synthesis and the FFTs,
 * orders m for the Legendre analysis, so no two threads write the same
 * coefficient. SHT_CPU_THREADS overrides the thread count.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

typedef struct { float re, im; } cf;

typedef struct {
    int grid, nh, nlat, lmax, mmax, nlayers;
    int64_t npoints, nlm;
    int *nlon, *mt;            /* nlon per northern ring, mmax_truncation */
    int64_t *ring_n, *ring_s;  /* first point of northern / southern ring j */
    int64_t *lm_off;           /* per m */
    float *lam;                /* [j][nlm] FP32 (legendre_polynomials[:, j]) */
    float *domega, *coslat_inv;
    cf **tw;                   /* per ring: exp(-2 pi i t / n), t < n */
    int **fac;                 /* per ring: factor list, fac[0] = count */
    int nfreq_max;
    double *x, *w;             /* Gaussian nodes (ascending) and weights */
} cpu_plan;

/* ---- a dynamic parallel-for over [0, n) on pthreads ---- */
static int g_threads = 0;
int cpu_max_threads(void) {
    if (g_threads <= 0) {
        const char* e = getenv("SHT_CPU_THREADS");
        g_threads = e ? atoi(e) : (int)sysconf(_SC_NPROCESSORS_ONLN);
        if (g_threads < 1) g_threads = 1;
        if (g_threads > 256) g_threads = 256;
    }
    return g_threads;
}
void cpu_set_threads(int n) { g_threads = n < 1 ? 1 : (n > 256 ? 256 : n); }

typedef void (*body_fn)(void* ctx, int i, int tid);
typedef struct { body_fn fn; void* ctx; int n, tid; int* next; pthread_mutex_t* mu; } worker_arg;

static void* worker(void* a_) {
    worker_arg* a = (worker_arg*)a_;
    for (;;) {
        pthread_mutex_lock(a->mu);
        int i = (*a->next)++;
        pthread_mutex_unlock(a->mu);
        if (i >= a->n) break;
        a->fn(a->ctx, i, a->tid);
    }
    return NULL;
}

static void par_for(int n, int T, body_fn fn, void* ctx) {
    if (T > n) T = n;
    if (T <= 1) { for (int i = 0; i < n; ++i) fn(ctx, i, 0); return; }
    pthread_t th[256];
    worker_arg args[256];
    int next = 0;
    pthread_mutex_t mu = PTHREAD_MUTEX_INITIALIZER;
    for (int t = 0; t < T; ++t) {
        args[t].fn = fn; args[t].ctx = ctx; args[t].n = n; args[t].tid = t; args[t].next = &next; args[t].mu = &mu;
        pthread_create(&th[t], NULL, worker, &args[t]);
    }
    for (int t = 0; t < T; ++t) pthread_join(th[t], NULL);
}

static void gauss_legendre(int n, double* x, double* w) {
    for (int i = 0; i < (n + 1) / 2; ++i) {
        double z = cos(M_PI * (i + 0.75) / (n + 0.5)), dp = 1, p0, p1;
        for (int it = 0; it < 100; ++it) {
            p0 = 1; p1 = z;
            for (int k = 2; k <= n; ++k) { double p2 = ((2.0 * k - 1) * z * p1 - (k - 1.0) * p0) / k; p0 = p1; p1 = p2; }
            dp = n * (z * p1 - p0) / (z * z - 1);
            double dz = p1 / dp; z -= dz;
            if (fabs(dz) < 1e-16) break;
        }
        p0 = 1; p1 = z;
        for (int k = 2; k <= n; ++k) { double p2 = ((2.0 * k - 1) * z * p1 - (k - 1.0) * p0) / k; p0 = p1; p1 = p2; }
        dp = n * (z * p1 - p0) / (z * z - 1);
        x[n - 1 - i] = z; x[i] = -z;
        w[n - 1 - i] = w[i] = 2.0 / ((1 - z * z) * dp * dp);
    }
}

static int* factorize(int n) {
    int tmp[64], c = 0, m = n;
    while (m % 4 == 0) { tmp[c++] = 4; m /= 4; }
    for (int p = 2; p * p <= m; ++p) while (m % p == 0) { tmp[c++] = p; m /= p; }
    if (m > 1) tmp[c++] = m;
    int* f = (int*)malloc((c + 1) * sizeof(int));
    f[0] = c;
    memcpy(f + 1, tmp, c * sizeof(int));
    return f;
}

static void plan_ring(void* ctx, int j, int tid) {
    (void)tid;
    cpu_plan* P = (cpu_plan*)ctx;
    const int lmax = P->lmax, mmax = P->mmax;
    double latd = acos(P->x[j]) * 180.0 / M_PI - 90.0;
    double colat = M_PI / 2 - latd * M_PI / 180.0;
    double xc = cos(colat), s = sqrt(fmax(0.0, 1 - xc * xc));
    int mt = P->nlon[j] / 2;                         /* LegendreShortcutLinear */
    P->mt[j] = mt < mmax - 1 ? mt : mmax - 1;
    P->domega[j] = (float)(P->w[j] * 2 * M_PI / P->nlon[j]);
    P->coslat_inv[j] = (float)(1.0 / cos(latd * M_PI / 180.0));
    double pmm = 1.0 / sqrt(4 * M_PI);
    float* L = P->lam + (size_t)j * P->nlm;
    for (int m = 0; m <= P->mt[j]; ++m) {
        if (m > 0) pmm = -sqrt((2.0 * m + 1) / (2.0 * m)) * s * pmm;
        float* col = L + P->lm_off[m];
        col[0] = (float)pmm;
        if (lmax - m >= 2) {
            double p0 = pmm, p1 = sqrt(2.0 * m + 3) * xc * pmm;
            double ap = sqrt((4.0 * (m + 1) * (m + 1) - 1) / ((m + 1.0) * (m + 1) - 1.0 * m * m));
            col[1] = (float)p1;
            for (int l = m + 2; l < lmax; ++l) {
                double a = sqrt((4.0 * l * l - 1) / (1.0 * l * l - 1.0 * m * m));
                double p2 = a * (xc * p1 - p0 / ap);
                col[l - m] = (float)p2;
                p0 = p1; p1 = p2; ap = a;
            }
        }
    }
    int n = P->nlon[j];
    P->tw[j] = (cf*)malloc(n * sizeof(cf));
    for (int t = 0; t < n; ++t) {
        P->tw[j][t].re = (float)cos(-2 * M_PI * t / n);
        P->tw[j][t].im = (float)sin(-2 * M_PI * t / n);
    }
    P->fac[j] = factorize(n);
}

void* cpu_plan_create(int grid, int nlat_half, int lmax, int mmax, int nlayers) {
    cpu_plan* P = (cpu_plan*)calloc(1, sizeof(cpu_plan));
    P->grid = grid; P->nh = nlat_half; P->nlat = 2 * nlat_half; P->lmax = lmax; P->mmax = mmax; P->nlayers = nlayers;
    int nh = P->nh;
    P->nlm = (int64_t)lmax * mmax - (int64_t)mmax * (mmax - 1) / 2;
    P->nlon = (int*)malloc(nh * sizeof(int));
    P->mt = (int*)malloc(nh * sizeof(int));
    P->ring_n = (int64_t*)malloc(nh * sizeof(int64_t));
    P->ring_s = (int64_t*)malloc(nh * sizeof(int64_t));
    int64_t off = 0;
    for (int j = 0; j < nh; ++j) {
        P->nlon[j] = grid == 0 ? 4 * nh : 16 + 4 * (j + 1);
        P->ring_n[j] = off; off += P->nlon[j];
    }
    for (int j = nh - 1; j >= 0; --j) { P->ring_s[j] = off; off += P->nlon[j]; }
    P->npoints = off;
    P->nfreq_max = 0;
    for (int j = 0; j < nh; ++j) if (P->nlon[j] / 2 + 1 > P->nfreq_max) P->nfreq_max = P->nlon[j] / 2 + 1;
    P->x = (double*)malloc(P->nlat * sizeof(double));
    P->w = (double*)malloc(P->nlat * sizeof(double));
    gauss_legendre(P->nlat, P->x, P->w);
    P->lm_off = (int64_t*)malloc(mmax * sizeof(int64_t));
    for (int m = 0; m < mmax; ++m) P->lm_off[m] = (int64_t)m * lmax - (int64_t)m * (m - 1) / 2;
    P->lam = (float*)calloc((size_t)nh * P->nlm, sizeof(float));
    P->domega = (float*)malloc(nh * sizeof(float));
    P->coslat_inv = (float*)malloc(nh * sizeof(float));
    P->tw = (cf**)malloc(nh * sizeof(cf*));
    P->fac = (int**)malloc(nh * sizeof(int*));
    par_for(nh, cpu_max_threads(), plan_ring, P);
    return P;
}

void cpu_plan_destroy(void* h) {
    cpu_plan* P = (cpu_plan*)h;
    if (!P) return;
    for (int j = 0; j < P->nh; ++j) { free(P->tw[j]); free(P->fac[j]); }
    free(P->tw); free(P->fac); free(P->nlon); free(P->mt); free(P->ring_n); free(P->ring_s); free(P->lm_off);
    free(P->lam); free(P->domega); free(P->coslat_inv); free(P->x); free(P->w); free(P);
}

int64_t cpu_npoints(void* h) { return ((cpu_plan*)h)->npoints; }
int64_t cpu_nlm(void* h) { return ((cpu_plan*)h)->nlm; }

/* y[k] = sum_t x[t] W^(+-k t), W = exp(-2 pi i / n): recursive mixed-radix decimation in time */
static void fft_rec(const cf* x, int xs, cf* y, int n, const int* fac, const cf* W, int ws, int inv, cf* tmp) {
    if (n == 1) { y[0] = x[0]; return; }
    int p = fac[0], m = n / p;
    for (int q = 0; q < p; ++q) fft_rec(x + q * xs, xs * p, y + q * m, m, fac + 1, W, ws * p, inv, tmp);
    for (int k = 0; k < m; ++k) {
        for (int q = 0; q < p; ++q) tmp[q] = y[q * m + k];
        for (int r = 0; r < p; ++r) {
            int idx = k + r * m;
            float sr = 0.f, si = 0.f;
            for (int q = 0; q < p; ++q) {
                int t = (int)(((int64_t)q * idx) % n);
                cf w = W[(int64_t)t * ws];
                float wi = inv ? -w.im : w.im;
                sr += tmp[q].re * w.re - tmp[q].im * wi;
                si += tmp[q].re * wi + tmp[q].im * w.re;
            }
            y[idx].re = sr; y[idx].im = si;
        }
    }
}

typedef struct {
    cpu_plan* P;
    const cf* coeffs;
    float* grid;
    int K, unscale;
    cf* work;         /* per thread: 2 * nfreq_max * K + 3 * (2 nfreq_max + 2) */
    size_t work_stride;
} syn_ctx;

static void syn_ring(void* ctx_, int j, int tid) {
    syn_ctx* c = (syn_ctx*)ctx_;
    cpu_plan* P = c->P;
    const int K = c->K, nf = P->nfreq_max, nmax = 2 * nf + 2;
    cf* gn = c->work + (size_t)tid * c->work_stride;
    cf* gs = gn + (size_t)nf * K;
    cf* z = gs + (size_t)nf * K;
    cf* y = z + nmax;
    cf* tmp = y + nmax;
    const float* L = P->lam + (size_t)j * P->nlm;
    memset(gn, 0, (size_t)nf * K * sizeof(cf));
    memset(gs, 0, (size_t)nf * K * sizeof(cf));
    const float sc = c->unscale ? P->coslat_inv[j] : 1.f;
    for (int m = 0; m <= P->mt[j]; ++m) {
        const float* lc = L + P->lm_off[m];
        const int len = P->lmax - m;
        for (int k = 0; k < K; ++k) {
            const cf* a = c->coeffs + (size_t)k * P->nlm + P->lm_off[m];
            float er = 0, ei = 0, or_ = 0, oi = 0;
            int l = 0;
            for (; l + 1 < len; l += 2) {
                er = fmaf(a[l].re, lc[l], er); ei = fmaf(a[l].im, lc[l], ei);
                or_ = fmaf(a[l + 1].re, lc[l + 1], or_); oi = fmaf(a[l + 1].im, lc[l + 1], oi);
            }
            if (l < len) { er = fmaf(a[l].re, lc[l], er); ei = fmaf(a[l].im, lc[l], ei); }
            gn[(size_t)k * nf + m].re = (er + or_) * sc; gn[(size_t)k * nf + m].im = (ei + oi) * sc;
            gs[(size_t)k * nf + m].re = (er - or_) * sc; gs[(size_t)k * nf + m].im = (ei - oi) * sc;
        }
    }
    const int n = P->nlon[j];
    for (int k = 0; k < K; ++k) {
        const cf* a = gn + (size_t)k * nf;
        const cf* b = gs + (size_t)k * nf;
        for (int mm = 0; mm <= n / 2; ++mm) {
            cf A = a[mm], B = b[mm];
            if (mm == 0 || 2 * mm == n) { A.im = 0; B.im = 0; }     /* c2r ignores Im of DC and Nyquist */
            z[mm].re = A.re - B.im; z[mm].im = A.im + B.re;
            if (mm > 0 && 2 * mm != n) { z[n - mm].re = A.re + B.im; z[n - mm].im = B.re - A.im; }
        }
        fft_rec(z, 1, y, n, P->fac[j] + 1, P->tw[j], 1, 1, tmp);
        float* gN = c->grid + (size_t)k * P->npoints + P->ring_n[j];
        float* gS = c->grid + (size_t)k * P->npoints + P->ring_s[j];
        for (int i = 0; i < n; ++i) { gN[i] = y[i].re; gS[i] = y[i].im; }
    }
}

/* coeffs: complex [K][nlm]; grid: [K][npoints] */
void cpu_synthesize(void* h, const float* coeffs, float* grid, int K, int unscale) {
    cpu_plan* P = (cpu_plan*)h;
    const int T = cpu_max_threads();
    syn_ctx c = {P, (const cf*)coeffs, grid, K, unscale, NULL, 0};
    c.work_stride = (size_t)2 * P->nfreq_max * K + 3 * (size_t)(2 * P->nfreq_max + 2);
    c.work = (cf*)malloc(c.work_stride * T * sizeof(cf));
    par_for(P->nh, T, syn_ring, &c);
    free(c.work);
}

typedef struct {
    cpu_plan* P;
    const float* grid;
    cf* coeffs;
    int K;
    cf *fe, *fo, *work;
    size_t work_stride;
} ana_ctx;

static void ana_ring(void* ctx_, int j, int tid) {
    ana_ctx* c = (ana_ctx*)ctx_;
    cpu_plan* P = c->P;
    const int K = c->K, nf = P->nfreq_max, nmax = 2 * nf + 2;
    cf* z = c->work + (size_t)tid * c->work_stride;
    cf* y = z + nmax;
    cf* tmp = y + nmax;
    const int n = P->nlon[j];
    const float dO = P->domega[j];
    for (int k = 0; k < K; ++k) {
        const float* gN = c->grid + (size_t)k * P->npoints + P->ring_n[j];
        const float* gS = c->grid + (size_t)k * P->npoints + P->ring_s[j];
        for (int i = 0; i < n; ++i) { z[i].re = gN[i]; z[i].im = gS[i]; }
        fft_rec(z, 1, y, n, P->fac[j] + 1, P->tw[j], 1, 0, tmp);
        cf* e = c->fe + ((size_t)j * K + k) * nf;
        cf* o = c->fo + ((size_t)j * K + k) * nf;
        for (int m = 0; m <= P->mt[j]; ++m) {
            cf a = y[m], b = y[m == 0 ? 0 : n - m];
            float fnr = 0.5f * (a.re + b.re), fni = 0.5f * (a.im - b.im);
            float fsr = 0.5f * (a.im + b.im), fsi = 0.5f * (b.re - a.re);
            e[m].re = dO * (fnr + fsr); e[m].im = dO * (fni + fsi);
            o[m].re = dO * (fnr - fsr); o[m].im = dO * (fni - fsi);
        }
    }
}

static void ana_order(void* ctx_, int m, int tid) {
    (void)tid;
    ana_ctx* c = (ana_ctx*)ctx_;
    cpu_plan* P = c->P;
    const int K = c->K, nf = P->nfreq_max, len = P->lmax - m;
    for (int k = 0; k < K; ++k) memset(c->coeffs + (size_t)k * P->nlm + P->lm_off[m], 0, len * sizeof(cf));
    for (int j = 0; j < P->nh; ++j) {
        if (m > P->mt[j]) continue;
        const float* lc = P->lam + (size_t)j * P->nlm + P->lm_off[m];
        for (int k = 0; k < K; ++k) {
            cf* a = c->coeffs + (size_t)k * P->nlm + P->lm_off[m];
            const cf ev = c->fe[((size_t)j * K + k) * nf + m], od = c->fo[((size_t)j * K + k) * nf + m];
            int l = 0;
            for (; l + 1 < len; l += 2) {
                a[l].re = fmaf(lc[l], ev.re, a[l].re); a[l].im = fmaf(lc[l], ev.im, a[l].im);
                a[l + 1].re = fmaf(lc[l + 1], od.re, a[l + 1].re); a[l + 1].im = fmaf(lc[l + 1], od.im, a[l + 1].im);
            }
            if (l < len) { a[l].re = fmaf(lc[l], ev.re, a[l].re); a[l].im = fmaf(lc[l], ev.im, a[l].im); }
        }
    }
}

void cpu_analyze(void* h, const float* grid, float* coeffs, int K) {
    cpu_plan* P = (cpu_plan*)h;
    const int T = cpu_max_threads(), nf = P->nfreq_max;
    ana_ctx c = {P, grid, (cf*)coeffs, K, NULL, NULL, NULL, 0};
    c.fe = (cf*)malloc((size_t)P->nh * K * nf * sizeof(cf));
    c.fo = (cf*)malloc((size_t)P->nh * K * nf * sizeof(cf));
    c.work_stride = 3 * (size_t)(2 * nf + 2);
    c.work = (cf*)malloc(c.work_stride * T * sizeof(cf));
    par_for(P->nh, T, ana_ring, &c);
    par_for(P->mmax, T, ana_order, &c);
    free(c.fe); free(c.fo); free(c.work);
}
