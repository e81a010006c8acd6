/*
 * fft3d.c -- the oracle's CPU FFT (test infrastructure only; see fft3d.h).
 *
 * Radix-2 iterative Cooley-Tukey for power-of-two lengths with twiddles taken
 * from long-double sin/cos (one rounding per twiddle), a direct DFT for other
 * lengths, and the two-for-one packing of two real rows into one complex
 * transform for the r2c/c2r axis. Strided axes are processed in blocks of
 * contiguous columns so every gather reads whole cache lines.
 */
#include "fft3d.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_COL_BLOCK 16

typedef struct {
    size_t n;
    int pow2;
    double* tw;     /* pow2: n/2 twiddles exp(-2 pi i k / n); else n twiddles */
    size_t* rev;    /* pow2 only: bit-reversal permutation */
} orc_plan1d;

static void plan_init(orc_plan1d* p, size_t n) {
    p->n = n;
    p->pow2 = n > 0 && (n & (n - 1)) == 0;
    const size_t ntw = p->pow2 ? (n / 2 > 0 ? n / 2 : 1) : n;
    p->tw = (double*)malloc(sizeof(double) * 2 * ntw);
    const long double two_pi = 6.283185307179586476925286766559005768L;
    for (size_t k = 0; k < ntw; ++k) {
        const long double ang = -two_pi * (long double)k / (long double)n;
        p->tw[2 * k] = (double)cosl(ang);
        p->tw[2 * k + 1] = (double)sinl(ang);
    }
    p->rev = NULL;
    if (p->pow2 && n > 1) {
        int bits = 0;
        while (((size_t)1 << bits) < n) ++bits;
        p->rev = (size_t*)malloc(sizeof(size_t) * n);
        for (size_t i = 0; i < n; ++i) {
            size_t r = 0;
            for (int b = 0; b < bits; ++b) r |= ((i >> b) & 1u) << (bits - 1 - b);
            p->rev[i] = r;
        }
    }
}

static void plan_free(orc_plan1d* p) {
    free(p->tw);
    free(p->rev);
}

/* In-place transform of one contiguous complex line; scratch holds n complex. */
static void plan_exec(const orc_plan1d* p, double* a, int sign, double* scratch) {
    const size_t n = p->n;
    if (n <= 1) return;
    if (p->pow2) {
        for (size_t i = 0; i < n; ++i) {
            const size_t j = p->rev[i];
            if (j > i) {
                double t0 = a[2 * i], t1 = a[2 * i + 1];
                a[2 * i] = a[2 * j]; a[2 * i + 1] = a[2 * j + 1];
                a[2 * j] = t0; a[2 * j + 1] = t1;
            }
        }
        for (size_t len = 2; len <= n; len <<= 1) {
            const size_t half = len >> 1;
            const size_t step = n / len;
            for (size_t i = 0; i < n; i += len) {
                for (size_t j = 0; j < half; ++j) {
                    const double wr = p->tw[2 * j * step];
                    const double wi = sign < 0 ? p->tw[2 * j * step + 1]
                                               : -p->tw[2 * j * step + 1];
                    double* u = a + 2 * (i + j);
                    double* v = a + 2 * (i + j + half);
                    const double vr = v[0] * wr - v[1] * wi;
                    const double vi = v[0] * wi + v[1] * wr;
                    v[0] = u[0] - vr; v[1] = u[1] - vi;
                    u[0] = u[0] + vr; u[1] = u[1] + vi;
                }
            }
        }
        return;
    }
    /* Direct DFT for non-power-of-two lengths. */
    for (size_t k = 0; k < n; ++k) {
        double sr = 0.0, si = 0.0;
        for (size_t j = 0; j < n; ++j) {
            const size_t t = (j * k) % n;
            const double wr = p->tw[2 * t];
            const double wi = sign < 0 ? p->tw[2 * t + 1] : -p->tw[2 * t + 1];
            sr += a[2 * j] * wr - a[2 * j + 1] * wi;
            si += a[2 * j] * wi + a[2 * j + 1] * wr;
        }
        scratch[2 * k] = sr;
        scratch[2 * k + 1] = si;
    }
    memcpy(a, scratch, sizeof(double) * 2 * n);
}

void orc_fft1d(size_t n, double* data, int sign) {
    orc_plan1d p;
    plan_init(&p, n);
    double* scratch = (double*)malloc(sizeof(double) * 2 * (n ? n : 1));
    plan_exec(&p, data, sign, scratch);
    free(scratch);
    plan_free(&p);
}

/* Transform the complex half-spectrum array c[N][N][H] along y (axis=1) or
 * x (axis=0), sign as in plan_exec. */
static void transform_strided_axis(size_t N, size_t H, double* c, int axis,
                                   int sign, const orc_plan1d* p) {
    const long long outer = (long long)N;
#pragma omp parallel
    {
        double* buf = (double*)malloc(sizeof(double) * 2 * N * ORC_COL_BLOCK);
        double* scratch = (double*)malloc(sizeof(double) * 2 * N);
#pragma omp for schedule(static)
        for (long long o = 0; o < outer; ++o) {
            for (size_t kz0 = 0; kz0 < H; kz0 += ORC_COL_BLOCK) {
                const size_t nb = (H - kz0) < ORC_COL_BLOCK ? (H - kz0) : ORC_COL_BLOCK;
                for (size_t i = 0; i < N; ++i) {
                    const size_t base = axis == 1
                        ? ((size_t)o * N + i) * H + kz0
                        : (i * N + (size_t)o) * H + kz0;
                    for (size_t b = 0; b < nb; ++b) {
                        buf[2 * (b * N + i)] = c[2 * (base + b)];
                        buf[2 * (b * N + i) + 1] = c[2 * (base + b) + 1];
                    }
                }
                for (size_t b = 0; b < nb; ++b) plan_exec(p, buf + 2 * b * N, sign, scratch);
                for (size_t i = 0; i < N; ++i) {
                    const size_t base = axis == 1
                        ? ((size_t)o * N + i) * H + kz0
                        : (i * N + (size_t)o) * H + kz0;
                    for (size_t b = 0; b < nb; ++b) {
                        c[2 * (base + b)] = buf[2 * (b * N + i)];
                        c[2 * (base + b) + 1] = buf[2 * (b * N + i) + 1];
                    }
                }
            }
        }
        free(buf);
        free(scratch);
    }
}

void orc_fft3d_r2c(size_t N, const double* in, double* out) {
    const size_t H = N / 2 + 1;
    const size_t rows = N * N;
    orc_plan1d p;
    plan_init(&p, N);
    /* z axis: two real rows per complex transform. */
    const long long pairs = (long long)((rows + 1) / 2);
#pragma omp parallel
    {
        double* z = (double*)malloc(sizeof(double) * 2 * N);
        double* scratch = (double*)malloc(sizeof(double) * 2 * N);
#pragma omp for schedule(static)
        for (long long q = 0; q < pairs; ++q) {
            const size_t ra = 2 * (size_t)q;
            const size_t rb = ra + 1;
            const int has_b = rb < rows;
            for (size_t k = 0; k < N; ++k) {
                z[2 * k] = in[ra * N + k];
                z[2 * k + 1] = has_b ? in[rb * N + k] : 0.0;
            }
            plan_exec(&p, z, -1, scratch);
            for (size_t k = 0; k < H; ++k) {
                const size_t m = (N - k) % N;
                const double zr = z[2 * k], zi = z[2 * k + 1];
                const double cr = z[2 * m], ci = -z[2 * m + 1];
                /* A = (Z[k] + conj Z[N-k]) / 2 ; B = (Z[k] - conj Z[N-k]) / (2i) */
                out[2 * (ra * H + k)] = 0.5 * (zr + cr);
                out[2 * (ra * H + k) + 1] = 0.5 * (zi + ci);
                if (has_b) {
                    out[2 * (rb * H + k)] = 0.5 * (zi - ci);
                    out[2 * (rb * H + k) + 1] = -0.5 * (zr - cr);
                }
            }
        }
        free(z);
        free(scratch);
    }
    transform_strided_axis(N, H, out, 1, -1, &p);
    transform_strided_axis(N, H, out, 0, -1, &p);
    plan_free(&p);
}

void orc_fft3d_c2r_destroy(size_t N, double* in, double* out) {
    const size_t H = N / 2 + 1;
    const size_t rows = N * N;
    orc_plan1d p;
    plan_init(&p, N);
    transform_strided_axis(N, H, in, 0, +1, &p);
    transform_strided_axis(N, H, in, 1, +1, &p);
    const long long pairs = (long long)((rows + 1) / 2);
#pragma omp parallel
    {
        double* z = (double*)malloc(sizeof(double) * 2 * N);
        double* scratch = (double*)malloc(sizeof(double) * 2 * N);
#pragma omp for schedule(static)
        for (long long q = 0; q < pairs; ++q) {
            const size_t ra = 2 * (size_t)q;
            const size_t rb = ra + 1;
            const int has_b = rb < rows;
            for (size_t k = 0; k < N; ++k) {
                double ar, ai, br = 0.0, bi = 0.0;
                const int conj_side = k >= H;
                const size_t src = conj_side ? N - k : k;
                ar = in[2 * (ra * H + src)];
                ai = in[2 * (ra * H + src) + 1];
                if (has_b) {
                    br = in[2 * (rb * H + src)];
                    bi = in[2 * (rb * H + src) + 1];
                }
                if (conj_side) { ai = -ai; bi = -bi; }
                if (k == 0 || (N % 2 == 0 && k == N / 2)) { ai = 0.0; bi = 0.0; }
                /* Z = A + i B */
                z[2 * k] = ar - bi;
                z[2 * k + 1] = ai + br;
            }
            plan_exec(&p, z, +1, scratch);
            for (size_t k = 0; k < N; ++k) {
                out[ra * N + k] = z[2 * k];
                if (has_b) out[rb * N + k] = z[2 * k + 1];
            }
        }
        free(z);
        free(scratch);
    }
    plan_free(&p);
}

void orc_fft3d_c2r(size_t N, const double* in_const, double* out) {
    /* Transform a private copy so the caller's half spectrum is untouched. */
    const size_t count = 2 * N * N * (N / 2 + 1);
    double* in = (double*)malloc(sizeof(double) * count);
    memcpy(in, in_const, sizeof(double) * count);
    orc_fft3d_c2r_destroy(N, in, out);
    free(in);
}
