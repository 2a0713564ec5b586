// Kernels of the learned WaveHoltz warm start: a Fourier neural operator (FNO) on a
// uniform G x G grid, trained and evaluated with BF16 operands and FP32 accumulation.
//
//   gemm        C = alpha op(A) op(B) + beta C, BF16 operands, FP32 accumulate and output,
//               batched with strides, optional split-K (atomic FP32 accumulation).  Tensor
//               cores through mma.sync.m16n8k16 (BF16): every GEMM of the network has one
//               dimension of 32 (channels or retained modes), so these are bandwidth-bound
//               streams, not tensor-throughput-bound tiles.
//   dft_y       the truncated DFT along y (retained wavenumbers 0..K/2-1 and -K/2..-1) and its
//               inverse/adjoint, FP32 on CUDA cores (small: K x KX modes per channel).
//   mix         per-mode complex channel mixing and its two adjoints.
//   pointwise   bias + GELU and its derivative, bias gradients, conversions, the MSE loss,
//               Adam, the resampling between the DG nodes and the grid, and the input
//               fields (forcing, omega, coordinates).
//
// The truncated DFT along x and the inverse real DFT along x are GEMMs against fixed
// BF16 matrices built by the host (fno.py).  All entry points are asynchronous on the
// given stream and return 0 or a negative WDG_ERR code.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "common.hpp"

namespace
{
    using bf16 = __nv_bfloat16;

    // ------------------------------------------------------------------ GEMM
    constexpr int TM = 64, TN = 64, TK = 32, LDS = TK + 8; // shared tiles: [64][40] bf16

    __device__ __forceinline__ void mma_bf16(float c[4], const uint32_t a[4], const uint32_t b[2])
    {
        asm volatile(
            "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
            "{%0,%1,%2,%3};"
            : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
            : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
    }

    struct GemmArgs
    {
        const bf16 *A, *B;
        float *C;
        int M, N, K;
        long long lda, ldb, ldc;       // leading dimensions of the stored matrices
        long long sA, sB, sC;          // batch strides (elements)
        int transA, transB;            // op(A)[m][k] = transA ? A[k*lda + m] : A[m*lda + k]
        float alpha, beta;
        int ksplit;                    // K range per split (multiple of TK)
        int atomic;                    // accumulate with atomics (split K, or batches sharing C)
    };

    // 64 x 64 output tile per CTA, 4 warps of 32 x 32, K in steps of 32 through shared memory
    __global__ void __launch_bounds__(128) gemm_bf16_kernel(const GemmArgs g)
    {
        __shared__ __align__(16) bf16 As[TM][LDS]; // (m, k)
        __shared__ __align__(16) bf16 Bs[TN][LDS]; // (n, k)
        const int bz = blockIdx.z;
        const int nsplit = (g.K + g.ksplit - 1) / g.ksplit;
        const int batch = bz / nsplit, split = bz - batch * nsplit;
        const bf16 *A = g.A + batch * g.sA;
        const bf16 *B = g.B + batch * g.sB;
        float *C = g.C + batch * g.sC;
        const int m0 = blockIdx.y * TM, n0 = blockIdx.x * TN;
        const int k_begin = split * g.ksplit, k_end = min(g.K, k_begin + g.ksplit);
        const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
        const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
        const int gid = lane >> 2, tig = lane & 3;
        float acc[2][4][4] = {};
        const bf16 zero = __float2bfloat16(0.f);

        for (int k0 = k_begin; k0 < k_end; k0 += TK)
        {
            // stage A tile (m, k) and B tile (n, k); the stored layout decides which index runs
            // fastest across threads so the global reads stay coalesced
            for (int i = t; i < TM * TK; i += 128)
            {
                int m, k;
                if (g.transA) { k = i / TM; m = i - k * TM; }
                else { m = i / TK; k = i - m * TK; }
                const int gm = m0 + m, gk = k0 + k;
                bf16 v = zero;
                if (gm < g.M && gk < k_end)
                    v = g.transA ? A[(long long)gk * g.lda + gm] : A[(long long)gm * g.lda + gk];
                As[m][k] = v;
            }
            for (int i = t; i < TN * TK; i += 128)
            {
                int n, k;
                if (g.transB) { n = i / TK; k = i - n * TK; }
                else { k = i / TN; n = i - k * TN; }
                const int gn = n0 + n, gk = k0 + k;
                bf16 v = zero;
                if (gn < g.N && gk < k_end)
                    v = g.transB ? B[(long long)gn * g.ldb + gk] : B[(long long)gk * g.ldb + gn];
                Bs[n][k] = v;
            }
            __syncthreads();
#pragma unroll
            for (int kk = 0; kk < TK; kk += 16)
            {
                uint32_t af[2][4], bfr[4][2];
#pragma unroll
                for (int mi = 0; mi < 2; ++mi)
                {
                    const int r = wm + 16 * mi + gid;
                    af[mi][0] = *reinterpret_cast<const uint32_t *>(&As[r][kk + 2 * tig]);
                    af[mi][1] = *reinterpret_cast<const uint32_t *>(&As[r + 8][kk + 2 * tig]);
                    af[mi][2] = *reinterpret_cast<const uint32_t *>(&As[r][kk + 2 * tig + 8]);
                    af[mi][3] = *reinterpret_cast<const uint32_t *>(&As[r + 8][kk + 2 * tig + 8]);
                }
#pragma unroll
                for (int ni = 0; ni < 4; ++ni)
                {
                    const int c = wn + 8 * ni + gid;
                    bfr[ni][0] = *reinterpret_cast<const uint32_t *>(&Bs[c][kk + 2 * tig]);
                    bfr[ni][1] = *reinterpret_cast<const uint32_t *>(&Bs[c][kk + 2 * tig + 8]);
                }
#pragma unroll
                for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                    for (int ni = 0; ni < 4; ++ni)
                        mma_bf16(acc[mi][ni], af[mi], bfr[ni]);
            }
            __syncthreads();
        }
        // epilogue: C = alpha acc + beta C (split-K: atomic accumulation, beta applied by split 0)
#pragma unroll
        for (int mi = 0; mi < 2; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                for (int h = 0; h < 4; ++h)
                {
                    const int r = m0 + wm + 16 * mi + gid + ((h >= 2) ? 8 : 0);
                    const int c = n0 + wn + 8 * ni + 2 * tig + (h & 1);
                    if (r >= g.M || c >= g.N)
                        continue;
                    float *p = C + (long long)r * g.ldc + c;
                    const float v = g.alpha * acc[mi][ni][h];
                    if (!g.atomic)
                        *p = (g.beta == 0.f) ? v : v + g.beta * *p;
                    else
                        atomicAdd(p, v);
                }
    }

    __global__ void scale_kernel(float *x, long long n, float s)
    {
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
            x[i] *= s;
    }

    int blocks(long long n, int threads = 256)
    {
        long long b = (n + threads - 1) / threads;
        return (int)(b < 148 * 32 ? (b < 1 ? 1 : b) : 148 * 32);
    }

    // ------------------------------------------------------------- DFT along y
    // out[bc, k, kx] = sum_y e^{s i 2 pi ky(k) y / G} in[bc, y, kx]   (forward: s = -1)
    // ky(k) = k for k < K/2, k - K otherwise; complex values as (re, im) pairs
    __global__ void dft_y_fwd_kernel(const float *in, float *out, const float *cs, const float *sn, int BC, int G,
                                     int K, int KX, float sign)
    {
        const long long total = (long long)BC * K * KX;
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x)
        {
            const int kx = (int)(i % KX);
            const int k = (int)((i / KX) % K);
            const long long bc = i / ((long long)KX * K);
            const int ky = (k < K / 2) ? k : k - K;
            const int step = ((ky % G) + G) % G;
            const float *src = in + bc * (long long)G * KX * 2 + 2 * kx;
            float re = 0.f, im = 0.f;
            int ph = 0;
            for (int y = 0; y < G; ++y)
            {
                const float c = cs[ph], s = sign * sn[ph];
                const float xr = src[(long long)y * KX * 2], xi = src[(long long)y * KX * 2 + 1];
                re += c * xr - s * xi;
                im += c * xi + s * xr;
                ph += step;
                if (ph >= G)
                    ph -= G;
            }
            out[2 * i] = re;
            out[2 * i + 1] = im;
        }
    }

    // out[bc, y, kx] = sum_k e^{s i 2 pi ky(k) y / G} in[bc, k, kx]; FP32 and/or BF16 output
    __global__ void dft_y_inv_kernel(const float *in, float *out, bf16 *outb, const float *cs, const float *sn, int BC,
                                     int G, int K, int KX, float sign)
    {
        const long long total = (long long)BC * G * KX;
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x)
        {
            const int kx = (int)(i % KX);
            const int y = (int)((i / KX) % G);
            const long long bc = i / ((long long)KX * G);
            const float *src = in + bc * (long long)K * KX * 2 + 2 * kx;
            float re = 0.f, im = 0.f;
            for (int k = 0; k < K; ++k)
            {
                const int ky = (k < K / 2) ? k : k - K;
                const int ph = (int)((((long long)ky * y) % G + G) % G);
                const float c = cs[ph], s = sign * sn[ph];
                const float xr = src[(long long)k * KX * 2], xi = src[(long long)k * KX * 2 + 1];
                re += c * xr - s * xi;
                im += c * xi + s * xr;
            }
            if (out)
            {
                out[2 * i] = re;
                out[2 * i + 1] = im;
            }
            if (outb)
            {
                outb[2 * i] = __float2bfloat16(re);
                outb[2 * i + 1] = __float2bfloat16(im);
            }
        }
    }

    // ------------------------------------------------------------- mode mixing
    // out[b, o, m] = sum_c R[c, o, m] x[b, c, m]   (complex; m runs over the retained modes)
    __global__ void mix_fwd_kernel(const float *R, const float *x, float *out, int Bn, int Cin, int Cout, int Mm)
    {
        const long long total = (long long)Bn * Cout * Mm;
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x)
        {
            const int m = (int)(i % Mm);
            const int o = (int)((i / Mm) % Cout);
            const int b = (int)(i / ((long long)Mm * Cout));
            float re = 0.f, im = 0.f;
            for (int c = 0; c < Cin; ++c)
            {
                const float *r = R + 2 * (((long long)c * Cout + o) * Mm + m);
                const float *v = x + 2 * (((long long)b * Cin + c) * Mm + m);
                re += r[0] * v[0] - r[1] * v[1];
                im += r[0] * v[1] + r[1] * v[0];
            }
            out[2 * i] = re;
            out[2 * i + 1] = im;
        }
    }
    // dx[b, c, m] = sum_o conj(R[c, o, m]) dy[b, o, m]
    __global__ void mix_bwd_x_kernel(const float *R, const float *dy, float *dx, int Bn, int Cin, int Cout, int Mm)
    {
        const long long total = (long long)Bn * Cin * Mm;
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x)
        {
            const int m = (int)(i % Mm);
            const int c = (int)((i / Mm) % Cin);
            const int b = (int)(i / ((long long)Mm * Cin));
            float re = 0.f, im = 0.f;
            for (int o = 0; o < Cout; ++o)
            {
                const float *r = R + 2 * (((long long)c * Cout + o) * Mm + m);
                const float *d = dy + 2 * (((long long)b * Cout + o) * Mm + m);
                re += r[0] * d[0] + r[1] * d[1];
                im += r[0] * d[1] - r[1] * d[0];
            }
            dx[2 * i] = re;
            dx[2 * i + 1] = im;
        }
    }
    // dR[c, o, m] (+)= sum_b dy[b, o, m] conj(x[b, c, m])
    __global__ void mix_bwd_w_kernel(const float *x, const float *dy, float *dR, int Bn, int Cin, int Cout, int Mm,
                                     int accumulate)
    {
        const long long total = (long long)Cin * Cout * Mm;
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x)
        {
            const int m = (int)(i % Mm);
            const int o = (int)((i / Mm) % Cout);
            const int c = (int)(i / ((long long)Mm * Cout));
            float re = 0.f, im = 0.f;
            for (int b = 0; b < Bn; ++b)
            {
                const float *v = x + 2 * (((long long)b * Cin + c) * Mm + m);
                const float *d = dy + 2 * (((long long)b * Cout + o) * Mm + m);
                re += d[0] * v[0] + d[1] * v[1];
                im += d[1] * v[0] - d[0] * v[1];
            }
            if (accumulate)
            {
                dR[2 * i] += re;
                dR[2 * i + 1] += im;
            }
            else
            {
                dR[2 * i] = re;
                dR[2 * i + 1] = im;
            }
        }
    }

    // ------------------------------------------------------------- pointwise
    __device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.f + erff(z * 0.70710678118654752f)); }
    __device__ __forceinline__ float gelu_grad(float z)
    {
        const float cdf = 0.5f * (1.f + erff(z * 0.70710678118654752f));
        const float pdf = 0.39894228040143268f * expf(-0.5f * z * z);
        return cdf + z * pdf;
    }

    // z[b, c, p] += bias[c]; y = act ? gelu(z) : z (BF16 and/or FP32 copies)
    __global__ void bias_act_kernel(float *z, const float *bias, bf16 *yb, float *yf, int Bn, int Cn, long long P,
                                    int act)
    {
        const long long total = (long long)Bn * Cn * P;
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x)
        {
            const int c = (int)((i / P) % Cn);
            const float v = z[i] + bias[c];
            z[i] = v;
            const float y = act ? gelu(v) : v;
            if (yb)
                yb[i] = __float2bfloat16(y);
            if (yf)
                yf[i] = y;
        }
    }
    // dz = dy * gelu'(z) (act) or dy; FP32 and BF16 copies
    __global__ void act_bwd_kernel(const float *dy, const float *z, float *dz, bf16 *dzb, long long n, int act)
    {
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        {
            const float v = act ? dy[i] * gelu_grad(z[i]) : dy[i];
            if (dz)
                dz[i] = v;
            if (dzb)
                dzb[i] = __float2bfloat16(v);
        }
    }
    // db[c] (+)= sum_{b, p} dz[b, c, p] in a fixed summation order, in two launches so that the
    // whole GPU reads dz: block (c, slice) sums its slice of every sample's plane into part,
    // then one thread per channel adds the slices in order
    constexpr int kBiasSlices = 64;
    __global__ void bias_grad_partial_kernel(const float *__restrict__ dz, float *__restrict__ part, int Bn, int Cn,
                                             long long P)
    {
        __shared__ float red[256];
        const int c = blockIdx.x, sl = blockIdx.y;
        const long long chunk = (P + gridDim.y - 1) / gridDim.y;
        const long long p0 = sl * chunk, p1 = (p0 + chunk < P) ? p0 + chunk : P;
        float s = 0.f;
        for (int b = 0; b < Bn; ++b)
        {
            const float *row = dz + ((long long)b * Cn + c) * P;
            for (long long p = p0 + threadIdx.x; p < p1; p += blockDim.x)
                s += row[p];
        }
        red[threadIdx.x] = s;
        __syncthreads();
        for (int h = blockDim.x / 2; h > 0; h >>= 1)
        {
            if ((int)threadIdx.x < h)
                red[threadIdx.x] += red[threadIdx.x + h];
            __syncthreads();
        }
        if (threadIdx.x == 0)
            part[(long long)c * gridDim.y + sl] = red[0];
    }
    __global__ void bias_grad_final_kernel(const float *__restrict__ part, float *db, int Cn, int S, int accumulate)
    {
        const int c = blockIdx.x * blockDim.x + threadIdx.x;
        if (c >= Cn)
            return;
        float s = 0.f;
        for (int k = 0; k < S; ++k)
            s += part[(long long)c * S + k];
        db[c] = accumulate ? db[c] + s : s;
    }
    __global__ void f32_to_bf16_kernel(const float *x, bf16 *y, long long n)
    {
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
            y[i] = __float2bfloat16(x[i]);
    }
    // per-sample sum of squared errors and the gradient of the mean over everything
    __global__ void mse_kernel(const float *y, const float *t, float *dy, double *sse, long long n, float inv_count)
    {
        __shared__ double red[256];
        double s = 0.0;
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        {
            const float d = y[i] - t[i];
            s += (double)d * d;
            dy[i] = 2.f * d * inv_count;
        }
        red[threadIdx.x] = s;
        __syncthreads();
        for (int h = blockDim.x / 2; h > 0; h >>= 1)
        {
            if ((int)threadIdx.x < h)
                red[threadIdx.x] += red[threadIdx.x + h];
            __syncthreads();
        }
        if (threadIdx.x == 0)
            atomicAdd(sse, red[0]);
    }
    __global__ void adam_kernel(float *p, const float *g, float *m, float *v, long long n, float lr, float b1, float b2,
                                float eps, float c1, float c2, float wd)
    {
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        {
            const float gi = g[i] + wd * p[i];
            const float mi = b1 * m[i] + (1.f - b1) * gi;
            const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
            m[i] = mi;
            v[i] = vi;
            p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        }
    }

    // ------------------------------------------------------- grid <-> DG nodes
    // Inputs of one sample on the G x G cell-centred grid of [-1, 1]^2:
    // (gaussian forcing / amplitude, omega / omega_ref, x, y)
    __global__ void fno_inputs_kernel(float *in, int G, double cx, double cy, double sigma, double w)
    {
        const long long P = (long long)G * G;
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < P; i += (long long)gridDim.x * blockDim.x)
        {
            const int ix = (int)(i % G), iy = (int)(i / G);
            const double x = -1.0 + (ix + 0.5) * 2.0 / G, y = -1.0 + (iy + 0.5) * 2.0 / G;
            const double r2 = (x - cx) * (x - cx) + (y - cy) * (y - cy);
            in[i] = (float)exp(-r2 / (2.0 * sigma * sigma));
            in[P + i] = (float)w;
            in[2 * P + i] = (float)x;
            in[3 * P + i] = (float)y;
        }
    }
    // Lagrange basis of the n GLL nodes at t (barycentric form, FP64)
    __device__ void lagrange(int n, const double *xn, const double *wb, double t, double *phi)
    {
        for (int j = 0; j < n; ++j)
            if (t == xn[j])
            {
                for (int k = 0; k < n; ++k)
                    phi[k] = (k == j) ? 1.0 : 0.0;
                return;
            }
        double s = 0.0;
        for (int j = 0; j < n; ++j)
        {
            phi[j] = wb[j] / (t - xn[j]);
            s += phi[j];
        }
        for (int j = 0; j < n; ++j)
            phi[j] /= s;
    }
    // DG field u(d, i, j, el) on a uniform ne x ne mesh of [-1, 1]^2 (element el = ex + ne ey)
    // -> grid values out[d, iy, ix] * scale (its element's polynomial, evaluated exactly)
    __global__ void nodes_to_grid_kernel(const double *u, float *out, int ne, int n, const double *xn, const double *wb,
                                         int G, float scale)
    {
        const long long P = (long long)G * G;
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < P; i += (long long)gridDim.x * blockDim.x)
        {
            const int ix = (int)(i % G), iy = (int)(i / G);
            const double x = -1.0 + (ix + 0.5) * 2.0 / G, y = -1.0 + (iy + 0.5) * 2.0 / G;
            const double h = 2.0 / ne;
            int ex = (int)((x + 1.0) / h), ey = (int)((y + 1.0) / h);
            ex = min(max(ex, 0), ne - 1);
            ey = min(max(ey, 0), ne - 1);
            const double xi = 2.0 * (x - (-1.0 + ex * h)) / h - 1.0, eta = 2.0 * (y - (-1.0 + ey * h)) / h - 1.0;
            double px[16], py[16];
            lagrange(n, xn, wb, xi, px);
            lagrange(n, xn, wb, eta, py);
            const double *e = u + (long long)(ex + ne * ey) * 3 * n * n;
            double acc[3] = {0, 0, 0};
            for (int b = 0; b < n; ++b)
                for (int a = 0; a < n; ++a)
                {
                    const double wgt = px[a] * py[b];
                    const double *q = e + 3 * (a + n * b);
                    acc[0] += wgt * q[0];
                    acc[1] += wgt * q[1];
                    acc[2] += wgt * q[2];
                }
            for (int d = 0; d < 3; ++d)
                out[d * P + i] = (float)(acc[d] * scale);
        }
    }
    // grid field g[d, iy, ix] (cell centres) -> DG nodes (bilinear, clamped at the border) * scale
    __global__ void grid_to_nodes_kernel(const float *g, double *u, int ne, int n, const double *xn, int G, double scale)
    {
        const long long total = (long long)ne * ne * n * n;
        const long long P = (long long)G * G;
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x)
        {
            const int node = (int)(i % (n * n));
            const int el = (int)(i / (n * n));
            const int a = node % n, b = node / n, ex = el % ne, ey = el / ne;
            const double h = 2.0 / ne;
            const double x = -1.0 + ex * h + 0.5 * h * (xn[a] + 1.0), y = -1.0 + ey * h + 0.5 * h * (xn[b] + 1.0);
            const double fx = (x + 1.0) * G / 2.0 - 0.5, fy = (y + 1.0) * G / 2.0 - 0.5;
            int x0 = (int)floor(fx), y0 = (int)floor(fy);
            double tx = fx - x0, ty = fy - y0;
            if (x0 < 0) { x0 = 0; tx = 0.0; }
            if (y0 < 0) { y0 = 0; ty = 0.0; }
            if (x0 >= G - 1) { x0 = G - 2; tx = 1.0; }
            if (y0 >= G - 1) { y0 = G - 2; ty = 1.0; }
            for (int d = 0; d < 3; ++d)
            {
                const float *p = g + d * P;
                const double v = (1 - tx) * (1 - ty) * p[(long long)y0 * G + x0] + tx * (1 - ty) * p[(long long)y0 * G + x0 + 1] +
                                 (1 - tx) * ty * p[(long long)(y0 + 1) * G + x0] + tx * ty * p[(long long)(y0 + 1) * G + x0 + 1];
                u[3 * i + d] = v * scale;
            }
        }
    }

    cudaStream_t st(void *s) { return static_cast<cudaStream_t>(s); }
    int done(const char *what)
    {
        const cudaError_t e = cudaGetLastError();
        return e == cudaSuccess ? WDG_OK : wdg::cuda_fail(e, what);
    }
} // namespace

extern "C"
{
    int wdg_fno_gemm(const void *A, const void *B, float *C, int M, int N, int K, long long lda, long long ldb,
                     long long ldc, long long strideA, long long strideB, long long strideC, int batch, int transA,
                     int transB, float alpha, float beta, int ksplit, void *stream)
    {
        if (!A || !B || !C || M < 1 || N < 1 || K < 1 || batch < 1 || ksplit < 0)
            return wdg::fail(WDG_ERR_ARG, "wdg_fno_gemm: bad arguments");
        GemmArgs g{};
        g.A = static_cast<const bf16 *>(A);
        g.B = static_cast<const bf16 *>(B);
        g.C = C;
        g.M = M;
        g.N = N;
        g.K = K;
        g.lda = lda;
        g.ldb = ldb;
        g.ldc = ldc;
        g.sA = strideA;
        g.sB = strideB;
        g.sC = strideC;
        g.transA = transA;
        g.transB = transB;
        g.alpha = alpha;
        g.beta = beta;
        g.ksplit = (ksplit > 0) ? ((ksplit + TK - 1) / TK) * TK : ((K + TK - 1) / TK) * TK;
        const int nsplit = (K + g.ksplit - 1) / g.ksplit;
        // split K, or a batch that sums into one C (stride 0): accumulate atomically, beta first
        g.atomic = (nsplit > 1 || (batch > 1 && strideC == 0)) ? 1 : 0;
        if (g.atomic && beta != 1.f)
        {
            if (beta != 0.f)
                return wdg::fail(WDG_ERR_ARG, "wdg_fno_gemm: atomic accumulation needs beta 0 or 1");
            const int nb = (strideC == 0) ? 1 : batch;
            for (int b = 0; b < nb; ++b)
                for (int r = 0; r < M; ++r)
                    if (cudaMemsetAsync(C + b * strideC + (long long)r * ldc, 0, sizeof(float) * N, st(stream)) !=
                        cudaSuccess)
                        return done("wdg_fno_gemm");
        }
        dim3 grid((N + TN - 1) / TN, (M + TM - 1) / TM, batch * nsplit);
        if (grid.y > 65535 || grid.z > 65535)
            return wdg::fail(WDG_ERR_ARG, "wdg_fno_gemm: problem too large for one launch");
        gemm_bf16_kernel<<<grid, 128, 0, st(stream)>>>(g);
        return done("wdg_fno_gemm");
    }

    int wdg_fno_dft_y(const float *in, float *out, void *out_bf16, const float *cos_tab, const float *sin_tab, int BC,
                      int G, int K, int KX, int inverse, float sign, void *stream)
    {
        if (!in || !cos_tab || !sin_tab || BC < 1 || G < 2 || K < 2 || (K & 1) || KX < 1 || (!out && !out_bf16))
            return wdg::fail(WDG_ERR_ARG, "wdg_fno_dft_y: bad arguments");
        if (!inverse)
        {
            if (!out)
                return wdg::fail(WDG_ERR_ARG, "wdg_fno_dft_y: the forward transform writes FP32");
            dft_y_fwd_kernel<<<blocks((long long)BC * K * KX), 256, 0, st(stream)>>>(in, out, cos_tab, sin_tab, BC, G, K,
                                                                                    KX, sign);
        }
        else
            dft_y_inv_kernel<<<blocks((long long)BC * G * KX), 256, 0, st(stream)>>>(
                in, out, static_cast<bf16 *>(out_bf16), cos_tab, sin_tab, BC, G, K, KX, sign);
        return done("wdg_fno_dft_y");
    }

    int wdg_fno_mix(const float *R, const float *x, float *out, int B, int Cin, int Cout, int modes, void *stream)
    {
        mix_fwd_kernel<<<blocks((long long)B * Cout * modes), 256, 0, st(stream)>>>(R, x, out, B, Cin, Cout, modes);
        return done("wdg_fno_mix");
    }
    int wdg_fno_mix_bwd(const float *R, const float *x, const float *dy, float *dx, float *dR, int B, int Cin, int Cout,
                        int modes, int accumulate, void *stream)
    {
        if (dx)
            mix_bwd_x_kernel<<<blocks((long long)B * Cin * modes), 256, 0, st(stream)>>>(R, dy, dx, B, Cin, Cout, modes);
        if (dR)
            mix_bwd_w_kernel<<<blocks((long long)Cin * Cout * modes), 256, 0, st(stream)>>>(x, dy, dR, B, Cin, Cout,
                                                                                            modes, accumulate);
        return done("wdg_fno_mix_bwd");
    }
    int wdg_fno_bias_act(float *z, const float *bias, void *y_bf16, float *y_f32, int B, int C, long long P, int act,
                         void *stream)
    {
        bias_act_kernel<<<blocks((long long)B * C * P), 256, 0, st(stream)>>>(z, bias, static_cast<bf16 *>(y_bf16),
                                                                               y_f32, B, C, P, act);
        return done("wdg_fno_bias_act");
    }
    int wdg_fno_act_bwd(const float *dy, const float *z, float *dz, void *dz_bf16, long long n, int act, void *stream)
    {
        act_bwd_kernel<<<blocks(n), 256, 0, st(stream)>>>(dy, z, dz, static_cast<bf16 *>(dz_bf16), n, act);
        return done("wdg_fno_act_bwd");
    }
    int wdg_fno_bias_grad(const float *dz, float *db, int B, int C, long long P, int accumulate, void *stream)
    {
        if (B < 1 || C < 1 || P < 1)
            return wdg::fail(WDG_ERR_ARG, "wdg_fno_bias_grad: empty shape");
        // the slices' partial sums in stream-ordered scratch
        float *part = nullptr;
        const cudaError_t e = cudaMallocAsync(reinterpret_cast<void **>(&part), sizeof(float) * C * kBiasSlices, st(stream));
        if (e != cudaSuccess)
            return wdg::cuda_fail(e, "cudaMallocAsync (wdg_fno_bias_grad)");
        bias_grad_partial_kernel<<<dim3(C, kBiasSlices), 256, 0, st(stream)>>>(dz, part, B, C, P);
        bias_grad_final_kernel<<<(C + 127) / 128, 128, 0, st(stream)>>>(part, db, C, kBiasSlices, accumulate);
        cudaFreeAsync(part, st(stream));
        return done("wdg_fno_bias_grad");
    }
    int wdg_fno_to_bf16(const float *x, void *y, long long n, void *stream)
    {
        f32_to_bf16_kernel<<<blocks(n), 256, 0, st(stream)>>>(x, static_cast<bf16 *>(y), n);
        return done("wdg_fno_to_bf16");
    }
    int wdg_fno_mse(const float *y, const float *t, float *dy, double *sse, long long n, float inv_count, void *stream)
    {
        mse_kernel<<<blocks(n), 256, 0, st(stream)>>>(y, t, dy, sse, n, inv_count);
        return done("wdg_fno_mse");
    }
    int wdg_fno_adam(float *p, const float *g, float *m, float *v, long long n, float lr, float beta1, float beta2,
                     float eps, int step, float weight_decay, void *stream)
    {
        if (step < 1)
            return wdg::fail(WDG_ERR_ARG, "wdg_fno_adam: steps count from 1");
        float c1 = 1.f, c2 = 1.f;
        for (int i = 0; i < step && i < 100000; ++i)
        {
            c1 *= beta1;
            c2 *= beta2;
        }
        adam_kernel<<<blocks(n), 256, 0, st(stream)>>>(p, g, m, v, n, lr, beta1, beta2, eps, 1.f - c1, 1.f - c2,
                                                       weight_decay);
        return done("wdg_fno_adam");
    }
    int wdg_fno_inputs(float *in, int G, double cx, double cy, double sigma, double w, void *stream)
    {
        fno_inputs_kernel<<<blocks((long long)G * G), 256, 0, st(stream)>>>(in, G, cx, cy, sigma, w);
        return done("wdg_fno_inputs");
    }
    int wdg_fno_nodes_to_grid(const double *u, float *out, int ne, int n, const double *gll_x, const double *gll_bw,
                              int G, float scale, void *stream)
    {
        if (n < 2 || n > 16)
            return wdg::fail(WDG_ERR_ARG, "wdg_fno_nodes_to_grid: 2..16 nodes per direction");
        nodes_to_grid_kernel<<<blocks((long long)G * G), 256, 0, st(stream)>>>(u, out, ne, n, gll_x, gll_bw, G, scale);
        return done("wdg_fno_nodes_to_grid");
    }
    int wdg_fno_grid_to_nodes(const float *g, double *u, int ne, int n, const double *gll_x, int G, double scale,
                              void *stream)
    {
        grid_to_nodes_kernel<<<blocks((long long)ne * ne * n * n), 256, 0, st(stream)>>>(g, u, ne, n, gll_x, G, scale);
        return done("wdg_fno_grid_to_nodes");
    }
}
