/*
 * Power-of-two complex FFT in double precision.  TEST INFRASTRUCTURE ONLY.
 *
 * The reference PM transforms run through cuFFT D2Z/Z2D
 * (cuda/cufft_wrapper.cu:56-78) on the GPU path and through rustfft 6.4.1
 * (third-party, not vendored; src/treepm/pm_grid.rs:132-271) on the CPU path.
 * Both compute the unnormalised DFT X[k] = sum_j x[j] exp(-2 pi i jk/n); this
 * file computes the same transform with an iterative radix-2 Cooley-Tukey
 * algorithm (bit reversal + butterflies, twiddles from cos/sin of the exact
 * angle), which agrees with either library to f64 rounding.
 */
#include "oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

void orc_fft1d(double* a, int n, int sign)
{
    /* bit-reversal permutation */
    for (int i = 1, j = 0; i < n; i++) {
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
        int half = len >> 1;
        for (int k = 0; k < half; k++) {
            double ang = sign * 2.0 * M_PI * (double)k / (double)len;
            double wr = cos(ang), wi = sin(ang);
            for (int s = 0; s < n; s += len) {
                double* u = a + 2 * (s + k);
                double* v = a + 2 * (s + k + half);
                double vr = v[0] * wr - v[1] * wi;
                double vi = v[0] * wi + v[1] * wr;
                v[0] = u[0] - vr; v[1] = u[1] - vi;
                u[0] += vr; u[1] += vi;
            }
        }
    }
}

void orc_fft3d(double* data, int M, int sign)
{
    int64_t M2 = (int64_t)M * M;
    /* x lines (contiguous) */
#pragma omp parallel for schedule(static)
    for (int64_t l = 0; l < M2; l++) orc_fft1d(data + 2 * l * M, M, sign);
    /* y and z lines (strided): gather, transform, scatter */
#pragma omp parallel
    {
        double* buf = (double*)malloc(sizeof(double) * 2 * M);
#pragma omp for schedule(static)
        for (int64_t l = 0; l < M2; l++) {
            int64_t x = l % M, z = l / M;
            for (int y = 0; y < M; y++) {
                int64_t idx = x + M * (y + (int64_t)M * z);
                buf[2 * y] = data[2 * idx]; buf[2 * y + 1] = data[2 * idx + 1];
            }
            orc_fft1d(buf, M, sign);
            for (int y = 0; y < M; y++) {
                int64_t idx = x + M * (y + (int64_t)M * z);
                data[2 * idx] = buf[2 * y]; data[2 * idx + 1] = buf[2 * y + 1];
            }
        }
#pragma omp for schedule(static)
        for (int64_t l = 0; l < M2; l++) {
            int64_t x = l % M, y = l / M;
            for (int z = 0; z < M; z++) {
                int64_t idx = x + M * (y + (int64_t)M * z);
                buf[2 * z] = data[2 * idx]; buf[2 * z + 1] = data[2 * idx + 1];
            }
            orc_fft1d(buf, M, sign);
            for (int z = 0; z < M; z++) {
                int64_t idx = x + M * (y + (int64_t)M * z);
                data[2 * idx] = buf[2 * z]; data[2 * idx + 1] = buf[2 * z + 1];
            }
        }
        free(buf);
    }
}
