/* wdg_fno.h -- kernels of the learned WaveHoltz warm start (a Fourier neural operator).
 *
 * The reference has no learned component; these entry points serve the warm start
 * that replaces WaveHoltz's zero initial iterate (examples/waveholtz2d.cpp:165) with a
 * network prediction, after which the reference's fixed-point loop runs unchanged.
 * All pointers are device memory; `stream` is a cudaStream_t (null: legacy default).
 * BF16 arrays are passed as void*.  Every call is asynchronous and returns 0 or a
 * negative WDG_ERR_* code (wdg_last_error() in wdg_b200.h gives the message).
 */
#ifndef WDG_FNO_H
#define WDG_FNO_H

#ifdef __cplusplus
extern "C" {
#endif

/* C[b] = alpha op(A[b]) op(B[b]) + beta C[b], BF16 operands, FP32 accumulate and output.
 * op(A)[m][k] = transA ? A[k lda + m] : A[m lda + k] (likewise B with (k, n)); batch b uses
 * A + b strideA etc.  ksplit > 0 splits K into pieces of that size; split K, or batches with
 * strideC == 0 (summing into one C), accumulate atomically and need beta 0 or 1. */
int wdg_fno_gemm(const void *A, const void *B, float *C, int M, int N, int K, long long lda, long long ldb,
                 long long ldc, long long strideA, long long strideB, long long strideC, int batch, int transA,
                 int transB, float alpha, float beta, int ksplit, void *stream);
/* DFT along y on the retained wavenumbers ky(k) = k (k < K/2), k - K (k >= K/2):
 * forward (inverse = 0): out[bc, k, kx] = sum_y e^{sign i 2 pi ky y / G} in[bc, y, kx];
 * inverse (inverse = 1): out[bc, y, kx] = sum_k e^{sign i 2 pi ky y / G} in[bc, k, kx]
 * (FP32 `out` and/or BF16 `out_bf16`).  Complex values are (re, im) pairs; cos_tab and
 * sin_tab hold cos / sin (2 pi m / G), m < G. */
int wdg_fno_dft_y(const float *in, float *out, void *out_bf16, const float *cos_tab, const float *sin_tab, int BC,
                  int G, int K, int KX, int inverse, float sign, void *stream);
/* per-mode complex channel mixing out[b, o, m] = sum_c R[c, o, m] x[b, c, m] and its adjoints
 * dx = conj(R) dy, dR (+)= sum_b dy conj(x) */
int wdg_fno_mix(const float *R, const float *x, float *out, int B, int Cin, int Cout, int modes, void *stream);
int wdg_fno_mix_bwd(const float *R, const float *x, const float *dy, float *dx, float *dR, int B, int Cin, int Cout,
                    int modes, int accumulate, void *stream);
/* z[b, c, p] += bias[c]; y = act ? GELU(z) : z (BF16 and/or FP32); dz = dy GELU'(z) or dy */
int wdg_fno_bias_act(float *z, const float *bias, void *y_bf16, float *y_f32, int B, int C, long long P, int act,
                     void *stream);
int wdg_fno_act_bwd(const float *dy, const float *z, float *dz, void *dz_bf16, long long n, int act, void *stream);
/* db[c] (+)= sum_{b, p} dz[b, c, p], fixed summation order */
int wdg_fno_bias_grad(const float *dz, float *db, int B, int C, long long P, int accumulate, void *stream);
int wdg_fno_to_bf16(const float *x, void *y, long long n, void *stream);
/* *sse += sum (y - t)^2 (FP64), dy = 2 (y - t) inv_count */
int wdg_fno_mse(const float *y, const float *t, float *dy, double *sse, long long n, float inv_count, void *stream);
/* Adam (bias-corrected, step counts from 1), optional decoupled weight decay */
int wdg_fno_adam(float *p, const float *g, float *m, float *v, long long n, float lr, float beta1, float beta2,
                 float eps, int step, float weight_decay, void *stream);
/* network inputs on the G x G cell-centred grid of [-1, 1]^2: (exp(-|x - c|^2 / 2 sigma^2),
 * w, x, y) as 4 planes */
int wdg_fno_inputs(float *in, int G, double cx, double cy, double sigma, double w, void *stream);
/* a DG field u(d, i, j, el) of a uniform ne x ne mesh of [-1, 1]^2 (n GLL nodes gll_x with
 * barycentric weights gll_bw) evaluated exactly on the grid: out[d, iy, ix] * scale ... */
int wdg_fno_nodes_to_grid(const double *u, float *out, int ne, int n, const double *gll_x, const double *gll_bw,
                          int G, float scale, void *stream);
/* ... and a grid field back to the nodes by bilinear interpolation (clamped at the border) */
int wdg_fno_grid_to_nodes(const float *g, double *u, int ne, int n, const double *gll_x, int G, double scale,
                          void *stream);

#ifdef __cplusplus
}
#endif

#endif /* WDG_FNO_H */
