/*
 * FFT behind the project's FFTW3 API shim (fftw3.h beside this file).  Test
 * infrastructure only: it lets the reference's own sources compile and run on
 * hosts without FFTW, so their outputs can pin the oracle and serve as the
 * CPU baseline.
 *
 * Algorithm (textbook, written from the mathematics):
 *  - complex DFT of power-of-two length: iterative radix-2 decimation in time
 *    with a bit-reversal permutation and a twiddle table computed with cos/sin
 *    of 2*pi*k/n;
 *  - complex DFT of any other length: direct O(n^2) sum with the exponent
 *    reduced modulo n (only reached when the target is shorter than one
 *    macro segment, so n is small);
 *  - real-to-complex of even length N: pack x[2k] + i*x[2k+1] into a complex
 *    sequence of length N/2, transform, and split the even/odd spectra;
 *    odd N falls back to the direct complex DFT;
 *  - complex-to-real: the inverse of that split (unnormalised, like FFTW).
 */
#include "fftw3.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

struct fsmeld_shim_plan_s {
    int n;          /* real length */
    int kind;       /* 0 = r2c, 1 = c2r */
    int half;       /* complex length used internally (n/2, or n when odd) */
    int pow2;       /* half is a power of two */
    double* tw_re;  /* exp(-2*pi*i*j/half), j < half/2 (power-of-two path) */
    double* tw_im;
    double* sp_re;  /* exp(-2*pi*i*k/n), k <= n/2 (even/odd split) */
    double* sp_im;
    double* work;   /* 2*half doubles */
    double* in;     /* plan-time buffers for fftw_execute */
    fftw_complex* cin;
    double* out;
    fftw_complex* cout;
};

static const double kTwoPi = 6.283185307179586476925286766559;

fftw_complex* fftw_alloc_complex(unsigned long n) {
    return (fftw_complex*)malloc(sizeof(fftw_complex) * (n ? n : 1));
}

double* fftw_alloc_real(unsigned long n) {
    return (double*)malloc(sizeof(double) * (n ? n : 1));
}

void fftw_free(void* p) { free(p); }

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

/* In-place complex DFT of length n (re/im interleaved in a), sign -1 or +1. */
static void cdft(const struct fsmeld_shim_plan_s* p, double* a, int n, int sign) {
    if (n <= 1) return;
    if (p->pow2) {
        /* bit reversal */
        for (int i = 1, j = 0; i < n; ++i) {
            int bit = n >> 1;
            for (; j & bit; bit >>= 1) j ^= bit;
            j ^= bit;
            if (i < j) {
                double tr = a[2 * i], ti = a[2 * i + 1];
                a[2 * i] = a[2 * j]; a[2 * i + 1] = a[2 * j + 1];
                a[2 * j] = tr; a[2 * j + 1] = ti;
            }
        }
        for (int len = 2; len <= n; len <<= 1) {
            const int stride = n / len;
            const int h = len >> 1;
            for (int s = 0; s < n; s += len) {
                for (int k = 0; k < h; ++k) {
                    const double wr = p->tw_re[k * stride];
                    const double wi = sign < 0 ? p->tw_im[k * stride] : -p->tw_im[k * stride];
                    double* u = a + 2 * (s + k);
                    double* v = a + 2 * (s + k + h);
                    const double xr = v[0] * wr - v[1] * wi;
                    const double xi = v[0] * wi + v[1] * wr;
                    v[0] = u[0] - xr; v[1] = u[1] - xi;
                    u[0] = u[0] + xr; u[1] = u[1] + xi;
                }
            }
        }
        return;
    }
    /* direct DFT */
    double* tmp = p->work + 2 * n;   /* work has room for 4*half doubles */
    for (int k = 0; k < n; ++k) {
        double sr = 0.0, si = 0.0;
        for (int j = 0; j < n; ++j) {
            const long long e = ((long long)j * k) % n;
            const double ang = kTwoPi * (double)e / (double)n;
            const double c = cos(ang), s = sign * sin(ang);
            sr += a[2 * j] * c - a[2 * j + 1] * s;
            si += a[2 * j] * s + a[2 * j + 1] * c;
        }
        tmp[2 * k] = sr; tmp[2 * k + 1] = si;
    }
    memcpy(a, tmp, sizeof(double) * 2 * n);
}

static struct fsmeld_shim_plan_s* make_plan(int n, int kind) {
    struct fsmeld_shim_plan_s* p = (struct fsmeld_shim_plan_s*)calloc(1, sizeof(*p));
    p->n = n;
    p->kind = kind;
    p->half = (n % 2 == 0) ? n / 2 : n;
    p->pow2 = is_pow2(p->half);
    const int h = p->half;
    p->tw_re = (double*)malloc(sizeof(double) * (h / 2 + 1));
    p->tw_im = (double*)malloc(sizeof(double) * (h / 2 + 1));
    for (int j = 0; j <= h / 2; ++j) {
        const double ang = kTwoPi * (double)j / (double)h;
        p->tw_re[j] = cos(ang);
        p->tw_im[j] = -sin(ang);
    }
    p->sp_re = (double*)malloc(sizeof(double) * (n / 2 + 1));
    p->sp_im = (double*)malloc(sizeof(double) * (n / 2 + 1));
    for (int k = 0; k <= n / 2; ++k) {
        const double ang = kTwoPi * (double)k / (double)n;
        p->sp_re[k] = cos(ang);
        p->sp_im[k] = -sin(ang);
    }
    p->work = (double*)malloc(sizeof(double) * 4 * (h + 1));
    return p;
}

fftw_plan fftw_plan_dft_r2c_1d(int n, double* in, fftw_complex* out, unsigned flags) {
    (void)flags;
    struct fsmeld_shim_plan_s* p = make_plan(n, 0);
    p->in = in; p->cout = out;
    return p;
}

fftw_plan fftw_plan_dft_c2r_1d(int n, fftw_complex* in, double* out, unsigned flags) {
    (void)flags;
    struct fsmeld_shim_plan_s* p = make_plan(n, 1);
    p->cin = in; p->out = out;
    return p;
}

void fftw_execute_dft_r2c(const fftw_plan p, double* in, fftw_complex* out) {
    const int n = p->n;
    double* z = p->work;
    if (n % 2) {
        for (int j = 0; j < n; ++j) { z[2 * j] = in[j]; z[2 * j + 1] = 0.0; }
        cdft(p, z, n, -1);
        for (int k = 0; k <= n / 2; ++k) { out[k][0] = z[2 * k]; out[k][1] = z[2 * k + 1]; }
        return;
    }
    const int h = n / 2;
    for (int j = 0; j < h; ++j) { z[2 * j] = in[2 * j]; z[2 * j + 1] = in[2 * j + 1]; }
    cdft(p, z, h, -1);
    for (int k = 0; k <= h; ++k) {
        const int a = k % h, b = (h - k) % h;
        const double zr = z[2 * a], zi = z[2 * a + 1];
        const double cr = z[2 * b], ci = -z[2 * b + 1];          /* conj(Z[h-k]) */
        const double er = 0.5 * (zr + cr), ei = 0.5 * (zi + ci); /* even spectrum */
        const double dr = 0.5 * (zr - cr), di = 0.5 * (zi - ci);
        const double orr = di, oi = -dr;                         /* odd = d / i */
        const double wr = p->sp_re[k], wi = p->sp_im[k];
        out[k][0] = er + (orr * wr - oi * wi);
        out[k][1] = ei + (orr * wi + oi * wr);
    }
}

void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex* in, double* out) {
    const int n = p->n;
    double* z = p->work;
    if (n % 2) {
        /* rebuild the full Hermitian spectrum, inverse DFT, keep real part */
        for (int k = 0; k < n; ++k) {
            if (k <= n / 2) { z[2 * k] = in[k][0]; z[2 * k + 1] = in[k][1]; }
            else { z[2 * k] = in[n - k][0]; z[2 * k + 1] = -in[n - k][1]; }
        }
        cdft(p, z, n, +1);
        for (int j = 0; j < n; ++j) out[j] = z[2 * j];
        return;
    }
    const int h = n / 2;
    for (int k = 0; k < h; ++k) {
        const double xr = in[k][0], xi = in[k][1];
        const double yr = in[h - k][0], yi = -in[h - k][1];     /* X[k+h] = conj(X[h-k]) */
        const double er = xr + yr, ei = xi + yi;
        const double dr = xr - yr, di = xi - yi;
        const double wr = p->sp_re[k], wi = -p->sp_im[k];       /* exp(+2*pi*i*k/n) */
        const double orr = dr * wr - di * wi, oi = dr * wi + di * wr;
        z[2 * k] = er - oi;                                      /* E + i*O */
        z[2 * k + 1] = ei + orr;
    }
    cdft(p, z, h, +1);
    for (int j = 0; j < h; ++j) { out[2 * j] = z[2 * j]; out[2 * j + 1] = z[2 * j + 1]; }
}

void fftw_execute(const fftw_plan p) {
    if (p->kind == 0) fftw_execute_dft_r2c(p, p->in, p->cout);
    else fftw_execute_dft_c2r(p, p->cin, p->out);
}

void fftw_destroy_plan(fftw_plan p) {
    if (!p) return;
    free(p->tw_re); free(p->tw_im); free(p->sp_re); free(p->sp_im); free(p->work);
    free(p);
}
