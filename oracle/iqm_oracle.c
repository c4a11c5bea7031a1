/*
 * iqm_oracle.c -- CPU restatement of cadik/IQM's metric arithmetic.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or calls this file;
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it, as the reference that
 * GPU results are compared with.
 *
 * The same source is compiled twice:
 *   -DORACLE_F32  -> liboracle_f32.so : arithmetic in float, in the order the reference's GLSL
 *                                       shaders and C++ host code use (the "reference-faithful
 *                                       FP32 restatement" and the timed CPU baseline);
 *   (default)     -> liboracle_f64.so : the same steps in double (the FP64 accuracy oracle).
 *
 * Every function cites the reference file:line it restates (paths within cadik/IQM).
 * Parity status: the reference ships no tests, golden vectors or fixtures, and its GPU path
 * (Vulkan + glslc + an unvendored VkFFT) cannot be built or run here.  M-SVD's CPU stage is
 * pinned against OpenCV (the reference's own library, via cv2) by fixtures in tests/golden;
 * the SSIM, FSIM and FLIP restatements are pinned by known-answer properties only
 * ("parity unpinned" for those three beyond the properties).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>

#ifdef ORACLE_F32
typedef float real;
#define RSQRT(x) sqrtf(x)
#define REXP(x) expf(x)
#define RLOG(x) logf(x)
#define RPOW(x, y) powf((x), (y))
#define RATAN2(y, x) atan2f((y), (x))
#define RSIN(x) sinf(x)
#define RCOS(x) cosf(x)
#define RFABS(x) fabsf(x)
#define RCEIL(x) ceilf(x)
#define RFLOOR(x) floorf(x)
#define RCBRT_POW(x) powf((x), 1.0f / 3.0f)
#define ORACLE_NAME "f32"
#else
typedef double real;
#define RSQRT(x) sqrt(x)
#define REXP(x) exp(x)
#define RLOG(x) log(x)
#define RPOW(x, y) pow((x), (y))
#define RATAN2(y, x) atan2((y), (x))
#define RSIN(x) sin(x)
#define RCOS(x) cos(x)
#define RFABS(x) fabs(x)
#define RCEIL(x) ceil(x)
#define RFLOOR(x) floor(x)
#define RCBRT_POW(x) pow((x), 1.0 / 3.0)
#define ORACLE_NAME "f64"
#endif
#define R(x) ((real)(x))

/* GLSL sources define PI as 3.141592653589 (e.g. shaders/fsim/fsim_angular.glsl:9). */
#define GLSL_PI 3.141592653589

const char *oracle_precision(void) { return ORACLE_NAME; }

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* ========================================================================================== */
/* Complex FFT (stands in for VkFFT, which the reference calls at src/gpu/fsim/fsim.cpp:364,378) */
/* Mixed-radix decimation in time for any size; Bluestein for prime factors above 61.          */
/* Sign -1 forward (unnormalised), +1 inverse; the caller applies 1/N like VkFFT normalize=1.  */
/* ========================================================================================== */
typedef struct { real re, im; } cplx;

static int smallest_factor(int n) {
    if (n % 4 == 0) return 4;
    if (n % 2 == 0) return 2;
    for (int p = 3; p * p <= n; p += 2)
        if (n % p == 0) return p;
    return n;
}

static void fft_any(cplx *x, int n, int sign);

static void fft_bluestein(cplx *x, int n, int sign) {
    int m = 1;
    while (m < 2 * n - 1) m <<= 1;
    cplx *a = calloc((size_t)m, sizeof(cplx));
    cplx *b = calloc((size_t)m, sizeof(cplx));
    cplx *w = malloc((size_t)n * sizeof(cplx));
    for (int k = 0; k < n; k++) {
        long k2 = ((long)k * k) % (2L * n);
        double ang = M_PI * (double)k2 / (double)n;
        w[k].re = (real)cos(ang);
        w[k].im = (real)(sign * sin(ang));
    }
    for (int k = 0; k < n; k++) {
        /* a_k = x_k * w_k ; b_k = conj(w_k) */
        a[k].re = x[k].re * w[k].re - x[k].im * w[k].im;
        a[k].im = x[k].re * w[k].im + x[k].im * w[k].re;
        b[k].re = w[k].re;
        b[k].im = -w[k].im;
        if (k > 0) { b[m - k] = b[k]; }
    }
    fft_any(a, m, -1);
    fft_any(b, m, -1);
    for (int k = 0; k < m; k++) {
        cplx t = {a[k].re * b[k].re - a[k].im * b[k].im, a[k].re * b[k].im + a[k].im * b[k].re};
        a[k] = t;
    }
    fft_any(a, m, +1);
    real inv = R(1.0) / (real)m;
    for (int k = 0; k < n; k++) {
        real cr = a[k].re * inv, ci = a[k].im * inv;
        x[k].re = cr * w[k].re - ci * w[k].im;
        x[k].im = cr * w[k].im + ci * w[k].re;
    }
    free(a); free(b); free(w);
}

/* Out-of-place recursive step on a sub-problem of size n of a top-level transform of size N:
 * X[k] = sum_r W_n^{r k} * FFT_m(x_r)[k mod m], with W_n^t = tw[t * (N/n)] from the top table.
 * `out` (size n) receives the result; `scratch` (size n) is free working space. */
static void fft_rec(const cplx *in, long istride, cplx *out, int n, int sign, cplx *scratch,
                    const cplx *tw, int N) {
    if (n == 1) { out[0] = in[0]; return; }
    int p = smallest_factor(n);
    if (p == n && n > 61) {
        for (int k = 0; k < n; k++) out[k] = in[(long)k * istride];
        fft_bluestein(out, n, sign);
        return;
    }
    int m = n / p;
    long step = N / n;
    /* sub-transforms of the p decimated sequences, stored contiguously in scratch */
    for (int r = 0; r < p; r++)
        fft_rec(in + (long)r * istride, istride * p, scratch + (long)r * m, m, sign, out, tw, N);
    for (int k = 0; k < n; k++) {
        int km = k % m;
        real sr = 0, si = 0;
        for (int r = 0; r < p; r++) {
            cplx w = tw[(((long)r * k) % n) * step];
            cplx y = scratch[(long)r * m + km];
            sr += y.re * w.re - y.im * w.im;
            si += y.re * w.im + y.im * w.re;
        }
        out[k].re = sr;
        out[k].im = si;
    }
}

static void fft_any(cplx *x, int n, int sign) {
    if (n <= 1) return;
    cplx *out = malloc((size_t)n * sizeof(cplx));
    cplx *scr = malloc((size_t)n * sizeof(cplx));
    cplx *tw = malloc((size_t)n * sizeof(cplx));
    /* twiddles exp(sign * 2 pi i j / n), evaluated in double and rounded to `real` */
    for (int j = 0; j < n; j++) {
        double ang = 2.0 * M_PI * (double)j / (double)n;
        tw[j].re = (real)cos(ang);
        tw[j].im = (real)(sign * sin(ang));
    }
    fft_rec(x, 1, out, n, sign, scr, tw, n);
    memcpy(x, out, (size_t)n * sizeof(cplx));
    free(out); free(scr); free(tw);
}

/* 2D transform of a row-major w x h plane (x fastest, VkFFT size[0] = width). */
static void fft2(cplx *d, int w, int h, int sign) {
    #pragma omp parallel for schedule(static)
    for (int y = 0; y < h; y++) fft_any(d + (long)y * w, w, sign);
    #pragma omp parallel
    {
        cplx *col = malloc((size_t)h * sizeof(cplx));
        #pragma omp for schedule(static)
        for (int x = 0; x < w; x++) {
            for (int y = 0; y < h; y++) col[y] = d[(long)y * w + x];
            fft_any(col, h, sign);
            for (int y = 0; y < h; y++) d[(long)y * w + x] = col[y];
        }
        free(col);
    }
}

/* Test hook: 2D FFT on interleaved doubles, computed in this build's precision. */
void oracle_fft2(double *data, int w, int h, int sign, int normalize) {
    long n = (long)w * h;
    cplx *d = malloc((size_t)n * sizeof(cplx));
    for (long i = 0; i < n; i++) { d[i].re = (real)data[2 * i]; d[i].im = (real)data[2 * i + 1]; }
    fft2(d, w, h, sign);
    real s = normalize ? R(1.0) / (real)n : R(1.0);
    for (long i = 0; i < n; i++) { data[2 * i] = (double)(d[i].re * s); data[2 * i + 1] = (double)(d[i].im * s); }
    free(d);
}

/* ========================================================================================== */
/* SSIM                                                                                        */
/* ========================================================================================== */

/* shaders/ssim/ssim_lumapack.glsl:19-21 -- note 0.581 for green (sic) on unorm [0,1] */
static inline real ssim_luma(const uint8_t *p) {
    real r = (real)p[0] / R(255.0), g = (real)p[1] / R(255.0), b = (real)p[2] / R(255.0);
    return R(0.299) * r + R(0.581) * g + R(0.114) * b;
}

/*
 * SSIM map + MSSIM.
 *   luma:        shaders/ssim/ssim_lumapack.glsl:19-35
 *   means:       shaders/ssim/ssim_gaussinput.glsl:22-57 (window truncated at the border and
 *                renormalised by the sum of the in-image weights)
 *   variances:   shaders/ssim/ssim.glsl:25-79 (two-pass form around the centre mean, same window)
 *   pooling:     src/gpu/ssim/ssim.cpp:386-401 (x,y in [r, dim-r] inclusive, summed in double)
 * Returns MSSIM; writes the W*H map when `map` is not NULL.
 */
double oracle_ssim(const uint8_t *in, const uint8_t *ref, int w, int h, long row_bytes,
                   int ksize, double k1d, double k2d, double sigmad, float *map) {
    long n = (long)w * h;
    real *la = malloc(n * sizeof(real)), *lb = malloc(n * sizeof(real));
    real *ma = malloc(n * sizeof(real)), *mb = malloc(n * sizeof(real));
    real *sm = malloc(n * sizeof(real));
    real sigma = (real)sigmad, k1 = (real)k1d, k2 = (real)k2d;
    int half = (ksize - 1) / 2;
    real *wt = malloc((size_t)ksize * ksize * sizeof(real));
    for (int xo = -half; xo <= half; xo++)
        for (int yo = -half; yo <= half; yo++) {
            real dist = (real)(xo * xo) + (real)(yo * yo);
            /* pow(E, -(dist / (2 sigma^2))) with E = 2.71828182846 (ssim.glsl:25-28) */
            wt[(xo + half) * ksize + (yo + half)] =
                RPOW(R(2.71828182846), -(dist / (R(2.0) * (sigma * sigma))));
        }
    #pragma omp parallel for schedule(static)
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            la[(long)y * w + x] = ssim_luma(in + (long)y * row_bytes + 4L * x);
            lb[(long)y * w + x] = ssim_luma(ref + (long)y * row_bytes + 4L * x);
        }
    #pragma omp parallel for schedule(static)
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            real ta = 0, tb = 0, tw = 0;
            for (int xo = -half; xo <= half; xo++)
                for (int yo = -half; yo <= half; yo++) {
                    int xx = x + xo, yy = y + yo;
                    if (xx >= w || yy >= h || xx < 0 || yy < 0) continue;
                    real wgt = wt[(xo + half) * ksize + (yo + half)];
                    ta += la[(long)yy * w + xx] * wgt;
                    tb += lb[(long)yy * w + xx] * wgt;
                    tw += wgt;
                }
            ma[(long)y * w + x] = ta / tw;
            mb[(long)y * w + x] = tb / tw;
        }
    real c1 = k1 * k1, c2 = k2 * k2;
    #pragma omp parallel for schedule(static)
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            real mA = ma[(long)y * w + x], mB = mb[(long)y * w + x];
            real vA = 0, vB = 0, cv = 0, tw = 0;
            for (int xo = -half; xo <= half; xo++)
                for (int yo = -half; yo <= half; yo++) {
                    int xx = x + xo, yy = y + yo;
                    if (xx >= w || yy >= h || xx < 0 || yy < 0) continue;
                    real wgt = wt[(xo + half) * ksize + (yo + half)];
                    real da = la[(long)yy * w + xx] - mA, db = lb[(long)yy * w + xx] - mB;
                    vA += da * da * wgt;
                    vB += db * db * wgt;
                    cv += da * db * wgt;
                    tw += wgt;
                }
            vA /= tw; vB /= tw; cv /= tw;
            sm[(long)y * w + x] = ((R(2.0) * mA * mB + c1) * (R(2.0) * cv + c2)) /
                                  ((mA * mA + mB * mB + c1) * (vA + vB + c2));
        }
    double sum = 0;
    unsigned start = (unsigned)half, wend = (unsigned)(w - half), hend = (unsigned)(h - half);
    for (unsigned y = start; y <= hend; y++)
        for (unsigned x = start; x <= wend; x++) sum += (double)sm[(long)y * w + x];
    double res = sum / (double)((wend - start + 1) * (hend - start + 1));
    if (map)
        for (long i = 0; i < n; i++) map[i] = (float)sm[i];
    free(la); free(lb); free(ma); free(mb); free(sm); free(wt);
    return res;
}

/* ========================================================================================== */
/* FSIM / FSIMc                                                                                */
/* ========================================================================================== */

/* src/gpu/fsim/fsim.cpp:165-168 */
int oracle_fsim_downscale_factor(int w, int h) {
    int smaller = w < h ? w : h;
    int f = (int)round(smaller / 256.0);
    return f > 1 ? f : 1;
}

/* shaders/fsim/fsim_lowpassfilter.glsl:31-35 and the same lines in the log-Gabor/angular
 * shaders: the ifftshift-ed, size-normalised frequency coordinate of index i on an n grid. */
static inline real freq_coord(int i, int n) {
    int shifted = (i + n / 2) % n;
    return (real)(shifted - n / 2) / (real)n;
}

/* Per-size filter bank: H[o*4+s][p] = logGabor_s(p) * angular_o(p).
 *   lowpass:   shaders/fsim/fsim_lowpassfilter.glsl:21-42, cutoff 0.45 order 15
 *              (src/gpu/fsim/steps/fsim_lowpass_filter.cpp:44-45)
 *   log-Gabor: shaders/fsim/fsim_log_gabor.glsl:16-49 (minWaveLength 6, mult 2, sigmaOnf 0.55)
 *   angular:   shaders/fsim/fsim_angular.glsl:16-48 (4 orientations, dThetaOnSigma 1.2)
 *   product:   shaders/fsim/fsim_filter_combinations.glsl:24-57 (z = o*4 + s)            */
static void fsim_filters(int w, int h, real *H /* 16*w*h */) {
    long n = (long)w * h;
    #pragma omp parallel for schedule(static)
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            real sx = freq_coord(x, w), sy = freq_coord(y, h);
            real radius = RSQRT(sx * sx + sy * sy);
            real lp = R(1.0) / (R(1.0) + RPOW(radius / R(0.45), R(2.0) * R(15.0)));
            real lg[4];
            for (int s = 0; s < 4; s++) {
                real wavelength = R(6.0) * RPOW(R(2.0), (real)s);
                real freq = R(1.0) / wavelength;
                real lr = RLOG(radius / freq);
                real ls = RLOG(R(0.55));
                real v = REXP(-(lr * lr) / (R(2.0) * (ls * ls)));
                lg[s] = (x == 0 && y == 0) ? R(0.0) : v * lp;
            }
            real thetaSigma = R(GLSL_PI) / R(4.0) / R(1.2);
            real theta = RATAN2(-sy, sx);
            real st = RSIN(theta), ct = RCOS(theta);
            for (int o = 0; o < 4; o++) {
                real angle = ((real)o * R(GLSL_PI)) / R(4.0);
                real ds = st * RCOS(angle) - ct * RSIN(angle);
                real dc = ct * RCOS(angle) + st * RSIN(angle);
                real dtheta = RFABS(RATAN2(ds, dc));
                real a = REXP(-(dtheta * dtheta) / (R(2.0) * (thetaSigma * thetaSigma)));
                for (int s = 0; s < 4; s++) H[(long)(o * 4 + s) * n + (long)y * w + x] = lg[s] * a;
            }
        }
}

/* Test hook: the 16 filter planes (o*4+s major) for a w x h grid, as doubles. */
void oracle_fsim_filters(int w, int h, double *out) {
    long n = (long)w * h;
    real *H = malloc(16 * n * sizeof(real));
    fsim_filters(w, h, H);
    for (long i = 0; i < 16 * n; i++) out[i] = (double)H[i];
    free(H);
}

/* Per-size constants (none depends on the images):
 *   em[o]   = EM_n(o) = sum_p H[o*4+0](p)^2                 -- fsim_filter_combinations.cpp:76-134,
 *                                                              shaders/fsim/fsim_filter_noise.glsl
 *   an2[o]  = sum_{p<lim} sum_s (Re ifft(H[o*4+s]))^2 * N     -- shaders/fsim/fsim_mult_filters.glsl:37-45
 *   aiaj[o] = sum_{p<lim} sum_{i<j} Re_i * Re_j * N            -- shaders/fsim/fsim_mult_filters.glsl:47-58
 * lim = ceil(N/2) by default: the reference's shader writes only p < ceil(N/2) (x = 2*tid < N,
 * fsim_mult_filters.glsl:27-31) yet sums all N entries of buffers never cleared
 * (fsim_estimate_energy.cpp:76-90); fresh device memory reads as 0.  energy_full=1 sums all N. */
void oracle_fsim_constants(int w, int h, int energy_full, double *em, double *an2, double *aiaj) {
    long n = (long)w * h;
    real *H = malloc(16 * n * sizeof(real));
    fsim_filters(w, h, H);
    cplx *sp = malloc(16 * n * sizeof(cplx));
    for (long i = 0; i < 16 * n; i++) { sp[i].re = H[i]; sp[i].im = 0; }
    for (int z = 0; z < 16; z++) fft2(sp + z * n, w, h, +1);
    real inv = R(1.0) / (real)n;
    long lim = energy_full ? n : (n + 1) / 2;
    for (int o = 0; o < 4; o++) {
        double e = 0, a2 = 0, ax = 0;
        for (long p = 0; p < n; p++) { real v = H[(long)(o * 4) * n + p]; e += (double)(v * v); }
        for (long p = 0; p < lim; p++) {
            real re[4];
            for (int s = 0; s < 4; s++) re[s] = sp[(long)(o * 4 + s) * n + p].re * inv;
            real s2 = 0, sx = 0;
            for (int s = 0; s < 4; s++) s2 += re[s] * re[s] * (real)n;
            for (int i = 0; i < 3; i++)
                for (int j = i + 1; j < 4; j++) sx += re[i] * re[j] * (real)n;
            a2 += (double)s2;
            ax += (double)sx;
        }
        em[o] = e; an2[o] = a2; aiaj[o] = ax;
    }
    free(H); free(sp);
}

static int cmp_real(const void *a, const void *b) {
    real x = *(const real *)a, y = *(const real *)b;
    return (x > y) - (x < y);
}

/* YIQ (0..255 units) box downsample -- shaders/fsim/fsim_downsample.glsl:21-55.
 * plane layout: yiq[0]=I, yiq[1]=Q, yiq[2]=Y, each w2*h2. */
static void fsim_downsample(const uint8_t *img, long row_bytes, int w, int h, int F, int w2, int h2,
                            real *yiq) {
    long n2 = (long)w2 * h2;
    real scaler = (real)(F * F);
    #pragma omp parallel for schedule(static)
    for (int y = 0; y < h2; y++)
        for (int x = 0; x < w2; x++) {
            real sI = 0, sQ = 0, sY = 0;
            int xs = x * F - F / 2, ys = y * F - F / 2;
            for (int j = xs; j < xs + F; j++)
                for (int k = ys; k < ys + F; k++) {
                    if (j >= 0 && j < w && k >= 0 && k < h) {
                        const uint8_t *p = img + (long)k * row_bytes + 4L * j;
                        real r = (real)p[0] / R(255.0) * R(255.0);
                        real g = (real)p[1] / R(255.0) * R(255.0);
                        real b = (real)p[2] / R(255.0) * R(255.0);
                        sI += r * R(0.596) - g * R(0.274) - b * R(0.322);
                        sQ += r * R(0.211) - g * R(0.523) + b * R(0.312);
                        sY += r * R(0.299) + g * R(0.587) + b * R(0.114);
                    }
                }
            yiq[0 * n2 + (long)y * w2 + x] = sI / scaler;
            yiq[1 * n2 + (long)y * w2 + x] = sQ / scaler;
            yiq[2 * n2 + (long)y * w2 + x] = sY / scaler;
        }
}

/* shaders/fsim/fsim_gradientmap.glsl:16-57 (zero padding, /16, magnitude) */
static void fsim_gradient(const real *Y, int w, int h, real *g) {
    static const real vert[9] = {3, 0, -3, 10, 0, -10, 3, 0, -3};
    static const real hor[9] = {3, 10, 3, 0, 0, 0, -3, -10, -3};
    #pragma omp parallel for schedule(static)
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            real vs = 0, hs = 0;
            for (int j = -1; j < 2; j++)
                for (int k = -1; k < 2; k++) {
                    int px = x + j, py = y + k;
                    if (px >= 0 && px < w && py >= 0 && py < h) {
                        real v = Y[(long)py * w + px];
                        int idx = (j + 1) + (k + 1) * 3;
                        vs += v * vert[idx];
                        hs += v * hor[idx];
                    }
                }
            real a = vs / R(16.0), b = hs / R(16.0);
            g[(long)y * w + x] = RSQRT(a * a + b * b);
        }
}

/*
 * FSIM and FSIMc of one pair -- src/gpu/fsim/fsim.cpp:80-163 and the step classes it drives.
 * energy_full selects the Q7 variant (see oracle_fsim_constants).  Optional debug outputs:
 * pc (2*w2*h2 floats: PC of input then reference) and noise (8 noise powers) may be NULL.
 */
int oracle_fsim(const uint8_t *in, const uint8_t *ref, int w, int h, long row_bytes, int energy_full,
                double *fsim, double *fsimc, float *pc_out, double *noise_out) {
    int F = oracle_fsim_downscale_factor(w, h);
    int w2 = (int)roundf((float)w / (float)F), h2 = (int)roundf((float)h / (float)F);
    long n = (long)w2 * h2;
    real *yiq[2], *grad[2];
    for (int i = 0; i < 2; i++) { yiq[i] = malloc(3 * n * sizeof(real)); grad[i] = malloc(n * sizeof(real)); }
    fsim_downsample(in, row_bytes, w, h, F, w2, h2, yiq[0]);
    fsim_downsample(ref, row_bytes, w, h, F, w2, h2, yiq[1]);
    fsim_gradient(yiq[0] + 2 * n, w2, h2, grad[0]);
    fsim_gradient(yiq[1] + 2 * n, w2, h2, grad[1]);

    /* forward FFT of luma (fsim_extractluma.glsl + fsim.cpp:270-368) */
    cplx *spec = malloc(2 * n * sizeof(cplx));
    for (int i = 0; i < 2; i++)
        for (long p = 0; p < n; p++) { spec[i * n + p].re = yiq[i][2 * n + p]; spec[i * n + p].im = 0; }
    fft2(spec, w2, h2, -1);
    fft2(spec + n, w2, h2, -1);

    real *H = malloc(16 * n * sizeof(real));
    fsim_filters(w2, h2, H);
    double em[4], an2[4], aiaj[4];
    oracle_fsim_constants(w2, h2, energy_full, em, an2, aiaj);

    /* 32 filtered spectra, inverse transformed with 1/N (fsim.cpp:403-431, normalize=true) */
    cplx *eo = malloc(32 * n * sizeof(cplx));
    for (int i = 0; i < 2; i++)
        for (int z = 0; z < 16; z++) {
            cplx *dst = eo + (long)(i * 16 + z) * n;
            for (long p = 0; p < n; p++) {
                real hz = H[(long)z * n + p];
                dst[p].re = hz * spec[i * n + p].re;
                dst[p].im = hz * spec[i * n + p].im;
            }
            fft2(dst, w2, h2, +1);
            real inv = R(1.0) / (real)n;
            for (long p = 0; p < n; p++) { dst[p].re *= inv; dst[p].im *= inv; }
        }

    /* per-orientation amplitude sum and energy -- shaders/fsim/fsim_sum_filter_responses.glsl:23-84 */
    real *amp = malloc(8 * n * sizeof(real)), *energy = malloc(8 * n * sizeof(real));
    for (int i = 0; i < 2; i++)
        for (int o = 0; o < 4; o++) {
            #pragma omp parallel for schedule(static)
            for (long p = 0; p < n; p++) {
                real sA = 0, sE = 0, sO = 0;
                for (int s = 0; s < 4; s++) {
                    cplx v = eo[(long)(i * 16 + o * 4 + s) * n + p];
                    sA += RSQRT(v.re * v.re + v.im * v.im);
                    sE += v.re;
                    sO += v.im;
                }
                real xe = RSQRT(sE * sE + sO * sO) + R(0.0001);
                real mE = sE / xe, mO = sO / xe;
                real en = 0;
                for (int s = 0; s < 4; s++) {
                    cplx v = eo[(long)(i * 16 + o * 4 + s) * n + p];
                    en += v.re * mE + v.im * mO - RFABS(v.re * mO - v.im * mE);
                }
                amp[(long)(i * 4 + o) * n + p] = sA;
                energy[(long)(i * 4 + o) * n + p] = en;
            }
        }

    /* noise power -- shaders/fsim/fsim_pack_for_median.glsl:27-46,
     * src/gpu/fsim/steps/fsim_noise_power.cpp:193-203 (upper median v[N/2] of a full sort) */
    real np_[8];
    real *tmp = malloc(n * sizeof(real));
    for (int idx = 0; idx < 8; idx++) {
        int i = idx / 4, o = idx % 4;
        for (long p = 0; p < n; p++) {
            cplx v = eo[(long)(i * 16 + o * 4 + 0) * n + p];
            tmp[p] = v.re * v.re + v.im * v.im;
        }
        qsort(tmp, (size_t)n, sizeof(real), cmp_real);
        real median = tmp[n / 2];
        real mean = -median / (real)log(0.5);
        np_[idx] = mean / (real)em[o];
        if (noise_out) noise_out[idx] = (double)np_[idx];
    }
    free(tmp);

    /* phase congruency -- shaders/fsim/fsim_phase_congruency.glsl:26-65 */
    real *pc = malloc(2 * n * sizeof(real));
    for (int i = 0; i < 2; i++) {
        real T[4];
        for (int o = 0; o < 4; o++) {
            real npw = np_[o + 4 * i];
            real e2 = R(2.0) * npw * (real)an2[o] + R(4.0) * npw * (real)aiaj[o];
            real tau = RSQRT(e2 / R(2.0));
            real ene = tau * RSQRT(R(GLSL_PI) / R(2.0));
            real sig = RSQRT((R(2.0) - R(GLSL_PI) / R(2.0)) * (tau * tau));
            T[o] = (ene + R(2.0) * sig) / R(1.7);
        }
        for (long p = 0; p < n; p++) {
            real et = 0, at = 0;
            for (int o = 0; o < 4; o++) {
                real e = energy[(long)(i * 4 + o) * n + p] - T[o];
                et += e > 0 ? e : R(0.0);
                at += amp[(long)(i * 4 + o) * n + p];
            }
            pc[i * n + p] = et / at;
        }
    }
    if (pc_out)
        for (long p = 0; p < 2 * n; p++) pc_out[p] = (float)pc[p];

    /* similarity and pooling -- shaders/fsim/fsim_final_multiply.glsl:18-58,
     * src/gpu/fsim/steps/fsim_final_multiply.cpp:294-300 (sums in double here) */
    double s_pcm = 0, s_sim = 0, s_simc = 0;
    for (long p = 0; p < n; p++) {
        real pc1 = pc[p], pc2 = pc[n + p];
        real pcm = pc1 > pc2 ? pc1 : pc2;
        real pcsim = (R(2.0) * pc1 * pc2 + R(0.85)) / (pc1 * pc1 + pc2 * pc2 + R(0.85));
        real g1 = grad[0][p], g2 = grad[1][p];
        real gsim = (R(2.0) * g1 * g2 + R(160.0)) / (g1 * g1 + g2 * g2 + R(160.0));
        real i1 = yiq[0][p], i2 = yiq[1][p], q1 = yiq[0][n + p], q2 = yiq[1][n + p];
        real isim = (R(2.0) * i1 * i2 + R(200.0)) / (i1 * i1 + i2 * i2 + R(200.0));
        real qsim = (R(2.0) * q1 * q2 + R(200.0)) / (q1 * q1 + q2 * q2 + R(200.0));
        real sim = gsim * pcsim * pcm;
        real simc = gsim * pcsim * RPOW(RFABS(isim * qsim), R(0.03)) * pcm;
        s_pcm += (double)pcm; s_sim += (double)sim; s_simc += (double)simc;
    }
    *fsim = s_sim / s_pcm;
    *fsimc = s_simc / s_pcm;
    for (int i = 0; i < 2; i++) { free(yiq[i]); free(grad[i]); }
    free(spec); free(H); free(eo); free(amp); free(energy); free(pc);
    return 0;
}

/* ========================================================================================== */
/* FLIP (LDR)                                                                                   */
/* ========================================================================================== */

/* src/gpu/flip/flip.cpp:125 -- FLIPArguments holds floats (src/gpu/flip/flip.h:21-25), so the first
 * two operations are float arithmetic; the pi/180 factor is double. */
double oracle_flip_ppd(double res_x, double distance, double width) {
    float f = (float)distance * ((float)res_x / (float)width);
    return (double)f * (M_PI / 180.0);
}

/* GLSL mat3(...) is column-major and `v * M` dots v with each column:
 * RGB_TO_XYZ columns from shaders/flip/srgb_to_ycxcz.glsl:16-20 */
static void rgb_to_xyz(const real c[3], real o[3]) {
    static const double M[3][3] = {
        {10135552.0 / 24577794, 8788810.0 / 24577794, 4435075.0 / 24577794},
        {2613072.0 / 12288897, 8788810.0 / 12288897, 887015.0 / 12288897},
        {1425312.0 / 73733382, 8788810.0 / 73733382, 70074185.0 / 73733382}};
    for (int i = 0; i < 3; i++)
        o[i] = c[0] * (real)(float)M[i][0] + c[1] * (real)(float)M[i][1] + c[2] * (real)(float)M[i][2];
}
/* XYZ_TO_RGB columns -- shaders/flip/spatial_prefilter.glsl:20-24 */
static void xyz_to_rgb(const real c[3], real o[3]) {
    static const double M[3][3] = {{3.241003275, -1.537398934, -0.498615861},
                                   {-0.969224334, 1.875930071, 0.041554224},
                                   {0.055639423, -0.204011202, 1.057148933}};
    for (int i = 0; i < 3; i++)
        o[i] = c[0] * (real)(float)M[i][0] + c[1] * (real)(float)M[i][1] + c[2] * (real)(float)M[i][2];
}
static void white_xyz(real o[3]) { real one[3] = {1, 1, 1}; rgb_to_xyz(one, o); }

/* shaders/flip/srgb_to_ycxcz.glsl:22-57 */
static void srgb_to_ycxcz(const uint8_t *p, real out[3]) {
    real c[3], lin[3], xyz[3], wp[3];
    for (int i = 0; i < 3; i++) {
        c[i] = (real)p[i] / R(255.0);
        lin[i] = c[i] > R(0.04045) ? RPOW((c[i] + R(0.055)) / R(1.055), R(2.4)) : c[i] / R(12.92);
    }
    rgb_to_xyz(lin, xyz);
    white_xyz(wp);
    for (int i = 0; i < 3; i++) xyz[i] /= wp[i];
    out[0] = R(116) * xyz[1] - R(16);
    out[1] = R(500) * (xyz[0] - xyz[1]);
    out[2] = R(200) * (xyz[1] - xyz[2]);
}

/* shaders/flip/spatial_prefilter_horizontal.glsl:24-26 */
static inline real csf_gauss(real d, const real par[4]) {
    real pi = R(GLSL_PI);
    return par[0] * RSQRT(pi / par[1]) * REXP(-(pi * pi) * d / par[1]) +
           par[2] * RSQRT(pi / par[3]) * REXP(-(pi * pi) * d / par[3]);
}

/* linear RGB -> L*a*b* (shaders/flip/spatial_detection.glsl:26-43, also inlined in
 * shaders/flip/spatial_prefilter.glsl:83-96) */
static void xyzn_to_lab(const real xyz[3], real lab[3]) {
    real delta = R(6.0) / R(29.0), limit = R(0.008856), c[3];
    for (int i = 0; i < 3; i++)
        c[i] = xyz[i] > limit ? RCBRT_POW(xyz[i]) : xyz[i] / (R(3.0) * delta * delta) + R(4.0) / R(29.0);
    lab[0] = R(116.0) * c[1] - R(16.0);
    lab[1] = R(500.0) * (c[0] - c[1]);
    lab[2] = R(200.0) * (c[1] - c[2]);
}
static void linrgb_to_lab(const real rgb[3], real lab[3]) {
    real xyz[3], wp[3];
    rgb_to_xyz(rgb, xyz);
    white_xyz(wp);
    for (int i = 0; i < 3; i++) xyz[i] /= wp[i];
    xyzn_to_lab(xyz, lab);
}
/* shaders/flip/spatial_detection.glsl:21-24 */
static inline real hyab(const real a[3], const real b[3]) {
    real d0 = a[0] - b[0], d1 = a[1] - b[1], d2 = a[2] - b[2];
    return RFABS(d0) + RSQRT(d1 * d1 + d2 * d2);
}

/* Feature taps (g, edge, point), normalised: shaders/flip/feature_filter.glsl:17-38 and
 * shaders/flip/feature_filter_normalize.glsl:17-47 (one clean normalisation pass). */
int oracle_flip_feature_taps(double ppd, double *taps /* 3*K, may be NULL */) {
    int K = 2 * (int)ceil(3 * 0.5 * 0.082 * ppd) + 1; /* src/gpu/flip/flip.cpp:126 */
    if (!taps) return K;
    real ppdf = (real)(float)ppd;
    real sd = R(0.5) * R(0.082) * ppdf;
    int radius = (int)RCEIL(R(3.0) * sd);
    real *t = malloc(3 * K * sizeof(real));
    real pos[3] = {0, 0, 0}, neg[3] = {0, 0, 0};
    for (int x = 0; x < K; x++) {
        int xc = x - radius;
        real g = REXP(-((real)xc * (real)xc) / (R(2.0) * (sd * sd)));
        t[0 * K + x] = g;
        t[1 * K + x] = -(real)xc * g;
        t[2 * K + x] = ((real)xc * (real)xc / (sd * sd) - R(1.0)) * g;
        for (int c = 0; c < 3; c++) {
            real v = t[c * K + x];
            if (v > 0) pos[c] += v; else neg[c] += -v;
        }
    }
    for (int c = 0; c < 3; c++)
        for (int x = 0; x < K; x++) {
            real v = t[c * K + x];
            taps[c * K + x] = (double)(v > 0 ? v / pos[c] : v / neg[c]);
        }
    free(t);
    return K;
}

/*
 * FLIP error map and its mean.  Per-pixel value from shaders/flip/combine_error_maps.glsl:28
 * (the reference never reads it back or pools it: FLIPResult::mean_flip at src/gpu/flip/flip.h:17
 * is never assigned); the mean of that value is the score defined for this restatement.
 * Passes: srgb_to_ycxcz.glsl, feature_filter(_normalize).glsl, feature_filter_horizontal.glsl,
 * feature_detection.glsl, spatial_prefilter_horizontal.glsl, spatial_prefilter.glsl,
 * spatial_detection.glsl, combine_error_maps.glsl.
 */
double oracle_flip(const uint8_t *in, const uint8_t *ref, int w, int h, long row_bytes, double ppd,
                   float *map) {
    long n = (long)w * h;
    real ppdf = (real)(float)ppd;
    real *ycc = malloc(2 * 3 * n * sizeof(real));
    const uint8_t *imgs[2] = {in, ref};
    for (int z = 0; z < 2; z++) {
        #pragma omp parallel for schedule(static)
        for (int y = 0; y < h; y++)
            for (int x = 0; x < w; x++) {
                real o[3];
                srgb_to_ycxcz(imgs[z] + (long)y * row_bytes + 4L * x, o);
                for (int c = 0; c < 3; c++) ycc[((long)z * 3 + c) * n + (long)y * w + x] = o[c];
            }
    }
    /* feature taps */
    int K = oracle_flip_feature_taps(ppd, NULL);
    double *td = malloc(3 * K * sizeof(double));
    oracle_flip_feature_taps(ppd, td);
    real *tg = malloc(3 * K * sizeof(real));
    for (int i = 0; i < 3 * K; i++) tg[i] = (real)td[i];
    free(td);
    int hk = K / 2;
    /* horizontal feature pass -> (dx, ddx, value) */
    real *fh = malloc(2 * 3 * n * sizeof(real));
    for (int z = 0; z < 2; z++) {
        #pragma omp parallel for schedule(static)
        for (int y = 0; y < h; y++)
            for (int x = 0; x < w; x++) {
                real dx = 0, ddx = 0, val = 0;
                for (int j = -hk; j <= hk; j++) {
                    int ax = clampi(x - j, 0, w - 1);
                    int fx = j + hk;
                    real v = (ycc[((long)z * 3 + 0) * n + (long)y * w + ax] + R(16.0)) / R(116.0);
                    val += tg[0 * K + fx] * v;
                    dx += tg[1 * K + fx] * v;
                    ddx += tg[2 * K + fx] * v;
                }
                fh[((long)z * 3 + 0) * n + (long)y * w + x] = dx;
                fh[((long)z * 3 + 1) * n + (long)y * w + x] = ddx;
                fh[((long)z * 3 + 2) * n + (long)y * w + x] = val;
            }
    }
    /* vertical feature pass -> deltaE_f */
    real *def = malloc(n * sizeof(real));
    #pragma omp parallel for schedule(static)
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            real dI[2] = {0, 0}, dR[2] = {0, 0}, ddI[2] = {0, 0}, ddR[2] = {0, 0};
            for (int k = -hk; k <= hk; k++) {
                int ay = clampi(y - k, 0, h - 1);
                int fy = k + hk;
                long pi = (long)ay * w + x;
                real vi0 = fh[0 * n + pi], vi1 = fh[1 * n + pi], vi2 = fh[2 * n + pi];
                real vr0 = fh[3 * n + pi], vr1 = fh[4 * n + pi], vr2 = fh[5 * n + pi];
                real f0 = tg[0 * K + fy], f1 = tg[1 * K + fy], f2 = tg[2 * K + fy];
                dI[0] += vi0 * f0; dI[1] += vi2 * f1;
                dR[0] += vr0 * f0; dR[1] += vr2 * f1;
                ddI[0] += vi1 * f0; ddI[1] += vi2 * f2;
                ddR[0] += vr1 * f0; ddR[1] += vr2 * f2;
            }
            real ed = RFABS(RSQRT(dI[0] * dI[0] + dI[1] * dI[1]) - RSQRT(dR[0] * dR[0] + dR[1] * dR[1]));
            real pd = RFABS(RSQRT(ddI[0] * ddI[0] + ddI[1] * ddI[1]) - RSQRT(ddR[0] * ddR[0] + ddR[1] * ddR[1]));
            real scaler = R(1.0) / RSQRT(R(2.0));
            real diff = ed > pd ? ed : pd;
            def[(long)y * w + x] = RPOW(scaler * diff, R(0.5));
        }
    free(fh);
    /* CSF prefilter, horizontal (shaders/flip/spatial_prefilter_horizontal.glsl:28-64) */
    static const double lumaP[4] = {1.0, 0.0047, 0, 0.00001}, rgP[4] = {1.0, 0.0053, 0, 0.00001},
                        byP[4] = {34.1, 0.04, 13.5, 0.025};
    real par[3][4];
    for (int i = 0; i < 4; i++) { par[0][i] = (real)(float)lumaP[i]; par[1][i] = (real)(float)rgP[i]; par[2][i] = (real)(float)byP[i]; }
    int radius = (int)RCEIL(R(3.0) * RSQRT(R(0.04) / (R(2.0) * R(GLSL_PI) * R(GLSL_PI))) * ppdf);
    real deltaX = R(1.0) / ppdf;
    real *ch = malloc(2 * 3 * n * sizeof(real));
    for (int z = 0; z < 2; z++) {
        #pragma omp parallel for schedule(static)
        for (int y = 0; y < h; y++)
            for (int x = 0; x < w; x++) {
                real op[3] = {0, 0, 0}, tot[3] = {0, 0, 0};
                for (int j = -radius; j <= radius; j++) {
                    int ax = clampi(x - j, 0, w - 1);
                    real xx = (real)j * deltaX;
                    real d = xx * xx;
                    for (int c = 0; c < 3; c++) {
                        real fv = csf_gauss(d, par[c]);
                        op[c] += ycc[((long)z * 3 + c) * n + (long)y * w + ax] * fv;
                        tot[c] += fv;
                    }
                }
                for (int c = 0; c < 3; c++) ch[((long)z * 3 + c) * n + (long)y * w + x] = op[c] / tot[c];
            }
    }
    free(ycc);
    /* CSF prefilter, vertical + colour transforms (shaders/flip/spatial_prefilter.glsl:40-102) */
    real *lab = malloc(2 * 3 * n * sizeof(real));
    for (int z = 0; z < 2; z++) {
        #pragma omp parallel for schedule(static)
        for (int y = 0; y < h; y++)
            for (int x = 0; x < w; x++) {
                real op[3] = {0, 0, 0}, tot[3] = {0, 0, 0};
                for (int k = -radius; k <= radius; k++) {
                    int ay = clampi(y - k, 0, h - 1);
                    real yy = (real)k * deltaX;
                    real d = yy * yy;
                    for (int c = 0; c < 3; c++) {
                        real fv = csf_gauss(d, par[c]);
                        op[c] += ch[((long)z * 3 + c) * n + (long)ay * w + x] * fv;
                        tot[c] += fv;
                    }
                }
                for (int c = 0; c < 3; c++) op[c] /= tot[c];
                real yyv = (op[0] + R(16.0)) / R(116.0), cx = op[1] / R(500.0), cz = op[2] / R(200.0);
                real wp[3], xyz[3], rgb[3], l[3];
                white_xyz(wp);
                xyz[0] = (yyv + cx) * wp[0]; xyz[1] = yyv * wp[1]; xyz[2] = (yyv - cz) * wp[2];
                xyz_to_rgb(xyz, rgb);
                for (int c = 0; c < 3; c++) rgb[c] = rgb[c] < 0 ? R(0) : (rgb[c] > 1 ? R(1) : rgb[c]);
                rgb_to_xyz(rgb, xyz);
                for (int c = 0; c < 3; c++) xyz[c] /= wp[c];
                xyzn_to_lab(xyz, l);
                l[1] *= R(0.01) * l[0];
                l[2] *= R(0.01) * l[0];
                for (int c = 0; c < 3; c++) lab[((long)z * 3 + c) * n + (long)y * w + x] = l[c];
            }
    }
    free(ch);
    /* colour error (shaders/flip/spatial_detection.glsl:57-85) and combine
     * (shaders/flip/combine_error_maps.glsl:15-33) */
    real green[3] = {0, 1, 0}, blue[3] = {0, 0, 1}, hg[3], hb[3];
    linrgb_to_lab(green, hg); hg[1] *= R(0.01) * hg[0]; hg[2] *= R(0.01) * hg[0];
    linrgb_to_lab(blue, hb); hb[1] *= R(0.01) * hb[0]; hb[2] *= R(0.01) * hb[0];
    real cmax = RPOW(hyab(hg, hb), R(0.7));
    double sum = 0;
    #pragma omp parallel for schedule(static) reduction(+ : sum)
    for (long p = 0; p < n; p++) {
        real a[3] = {lab[0 * n + p], lab[1 * n + p], lab[2 * n + p]};
        real b[3] = {lab[3 * n + p], lab[4 * n + p], lab[5 * n + p]};
        real dE = RPOW(hyab(a, b), R(0.7));
        real pc = R(0.4), pt = R(0.95), pcc = pc * cmax;
        real dEc = dE < pcc ? (pt / pcc) * dE : pt + ((dE - pcc) / (cmax - pcc)) * (R(1.0) - pt);
        real v = RPOW(dEc, R(1.0) - def[p]);
        if (map) map[p] = (float)v;
        sum += (double)v;
    }
    free(lab); free(def);
    return sum / (double)n;
}

/* ========================================================================================== */
/* M-SVD                                                                                        */
/* ========================================================================================== */

/* cv::cvtColor(COLOR_RGB2GRAY) on 8-bit data, as called at src/gpu/svd/svd.cpp:56-59:
 * BT.601 weights 0.299/0.587/0.114 in 15-bit fixed point (9798, 19235, 3735; they sum to 2^15)
 * with a round-half-up descale -- the OpenCV 4.x integer path.  Pinned against cv2 4.13 by the
 * fixtures in tests/golden (exact on every tested pixel). */
unsigned oracle_gray_u8(unsigned r, unsigned g, unsigned b) {
    return (r * 9798u + g * 19235u + b * 3735u + (1u << 14)) >> 15;
}

/* Singular values of one 8x8 block, descending (cv::SVD(.., NO_UV).w at src/gpu/svd/svd.cpp:80-81).
 * One-sided (Hestenes) Jacobi: columns are rotated in `real`; column norms and inner products
 * are accumulated in double and drive the convergence test. */
void oracle_svd8(const float *blk /* row-major 8x8 */, float *sv) {
    real a[8][8]; /* a[c][r] : column c */
    double nrm[8];
    for (int r = 0; r < 8; r++)
        for (int c = 0; c < 8; c++) a[c][r] = (real)blk[r * 8 + c];
    for (int c = 0; c < 8; c++) {
        double s = 0;
        for (int r = 0; r < 8; r++) s += (double)a[c][r] * (double)a[c][r];
        nrm[c] = s;
    }
#ifdef ORACLE_F32
    const double eps = (double)FLT_EPSILON;
#else
    const double eps = DBL_EPSILON;
#endif
    for (int sweep = 0; sweep < 60; sweep++) {
        int changed = 0;
        for (int i = 0; i < 7; i++)
            for (int j = i + 1; j < 8; j++) {
                double p = 0;
                for (int r = 0; r < 8; r++) p += (double)a[i][r] * (double)a[j][r];
                double ai = nrm[i], aj = nrm[j];
                if (fabs(p) <= eps * sqrt(ai * aj)) continue;
                /* rotation zeroing the (i,j) inner product */
                double zeta = (aj - ai) / (2.0 * p);
                double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
                double cs = 1.0 / sqrt(1.0 + t * t), sn = cs * t;
                real c = (real)cs, s = (real)sn;
                double ni = 0, nj = 0;
                for (int r = 0; r < 8; r++) {
                    real xi = a[i][r], xj = a[j][r];
                    real yi = c * xi - s * xj;
                    real yj = s * xi + c * xj;
                    a[i][r] = yi; a[j][r] = yj;
                    ni += (double)yi * yi; nj += (double)yj * yj;
                }
                nrm[i] = ni; nrm[j] = nj;
                changed = 1;
            }
        if (!changed) break;
    }
    double s[8];
    for (int c = 0; c < 8; c++) {
        double q = 0;
        for (int r = 0; r < 8; r++) q += (double)a[c][r] * (double)a[c][r];
        s[c] = sqrt(q);
    }
    for (int i = 0; i < 8; i++)
        for (int j = i + 1; j < 8; j++)
            if (s[j] > s[i]) { double t = s[i]; s[i] = s[j]; s[j] = t; }
    for (int i = 0; i < 8; i++) sv[i] = (float)s[i];
}

static int cmp_float(const void *a, const void *b) {
    float x = *(const float *)a, y = *(const float *)b;
    return (x > y) - (x < y);
}

/*
 * M-SVD -- src/gpu/svd/svd.cpp:39-164 and shaders/svd/svd.glsl:24-54.
 *   blocks: only where x+8 < W and y+8 < H (svd.cpp:68,74); slot (y/8)*(W/8) + x/8;
 *           skipped slots stay 0 yet count in n = (W/8)*(H/8)
 *   D     : sqrt(sum_k (s_k - r_k)^2) per block (float, svd.glsl:41-52)
 *   score : sort ascending, median = D[n/2], msvd = sum |D - median| / n
 *           (float running sum in the FP32 build, as svd.cpp:140-151; double in the FP64 build)
 *   map   : D / max(D) ((W/8)*(H/8) floats, svd.cpp:153-161), when `map` is not NULL.
 */
double oracle_msvd(const uint8_t *in, const uint8_t *ref, int w, int h, long row_bytes, float *map,
                   float *dist_out) {
    int bw = w / 8, bh = h / 8;
    long nb = (long)bw * bh;
    float *D = calloc((size_t)(nb > 0 ? nb : 1), sizeof(float));
    #pragma omp parallel for schedule(dynamic)
    for (int y = 0; y < h; y += 8) {
        if (!(y + 8 < h)) continue;
        for (int x = 0; x + 8 < w; x += 8) {
            float bi[64], br[64], si[8], sr[8];
            for (int r = 0; r < 8; r++)
                for (int c = 0; c < 8; c++) {
                    const uint8_t *p = in + (long)(y + r) * row_bytes + 4L * (x + c);
                    const uint8_t *q = ref + (long)(y + r) * row_bytes + 4L * (x + c);
                    bi[r * 8 + c] = (float)oracle_gray_u8(p[0], p[1], p[2]);
                    br[r * 8 + c] = (float)oracle_gray_u8(q[0], q[1], q[2]);
                }
            oracle_svd8(bi, si);
            oracle_svd8(br, sr);
            real acc = 0;
            for (int k = 0; k < 8; k++) {
                real d = (real)si[k] - (real)sr[k];
                acc += d * d;
            }
            D[(long)(y / 8) * bw + (x / 8)] = (float)RSQRT(acc);
        }
    }
    if (dist_out) memcpy(dist_out, D, nb * sizeof(float));
    float *s = malloc((size_t)(nb > 0 ? nb : 1) * sizeof(float));
    memcpy(s, D, nb * sizeof(float));
    qsort(s, (size_t)nb, sizeof(float), cmp_float);
    float mid = s[nb / 2];
    real sum = 0;
    for (long i = 0; i < nb; i++) sum += RFABS((real)s[i] - (real)mid);
    double res = (double)(sum / (real)nb);
    if (map) {
        float mx = -INFINITY;
        for (long i = 0; i < nb; i++) mx = D[i] > mx ? D[i] : mx;
        for (long i = 0; i < nb; i++) map[i] = D[i] / mx;
    }
    free(D); free(s);
    return res;
}
