// Learned coarse-grid closure: a small MLP (96 -> 128 -> 128 -> 128 -> 48, GELU on the hidden
// layers) with BF16 weights and activations and FP32 accumulation, with its own inference,
// training-forward, backward, gradient-reduction and Adam kernels, plus the closure's feature
// extraction from a coarse state and the application of its correction to an RK stage.
//
// Matrix products run on the tensor cores with mma.sync.m16n8k16 (bf16 x bf16 -> f32).  A warp
// owns 16 samples; the accumulator fragment of one layer (rows g, g + 8; columns 2t, 2t + 1 of
// each 8-column tile, g = lane / 4, t = lane % 4) is exactly the A fragment of the next layer's
// 16-column k tiles, so the activations of a sample tile stay in registers through the network.
// Weights are read as 32-bit pairs from two layouts kept by the optimizer: [out][in] for the
// forward product and [in][out] for the backward product.  The weight-gradient product
// (H^T dZ, a reduction over samples) goes through shared memory.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "vlasov1d2v.h"

void vl_internal_set_error(const char *msg);

namespace {

constexpr int IN = 96, HID = 128, OUT = 48;
constexpr int NL = 4;                          // layers
constexpr int WARPS = 4, ROWS = 16 * WARPS;    // samples per CTA tile
__host__ __device__ constexpr int layer_in(int l) { return l == 0 ? IN : HID; }
__host__ __device__ constexpr int layer_out(int l) { return l == NL - 1 ? OUT : HID; }

struct MlpWeights {
    const __nv_bfloat16 *wf[NL];   // [out][in]
    const __nv_bfloat16 *wb[NL];   // [in][out]
    const float *bias[NL];         // [out]
};

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, "
        "{%8, %9}, {%0, %1, %2, %3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t *>(&v);
}

// GELU(x) = x Phi(x) and its derivative Phi(x) + x phi(x) (erf form)
__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_d(float x) {
    const float cdf = 0.5f * (1.0f + erff(x * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * __expf(-0.5f * x * x);
    return cdf + x * pdf;
}

// A fragments (bf16 pairs) of a 16 x K row tile from FP32 accumulator fragments of K/8 n tiles:
// k tile kk takes n tiles 2kk (a0, a1) and 2kk + 1 (a2, a3)
template <int K>
__device__ __forceinline__ void acc_to_a(const float (&acc)[K / 8][4], uint32_t (&a)[K / 16][4]) {
#pragma unroll
    for (int kk = 0; kk < K / 16; ++kk) {
        a[kk][0] = pack_bf16(acc[2 * kk][0], acc[2 * kk][1]);
        a[kk][1] = pack_bf16(acc[2 * kk][2], acc[2 * kk][3]);
        a[kk][2] = pack_bf16(acc[2 * kk + 1][0], acc[2 * kk + 1][1]);
        a[kk][3] = pack_bf16(acc[2 * kk + 1][2], acc[2 * kk + 1][3]);
    }
}

// acc[n tile][4] = A (16 x K, fragments) . W (K x N), W given as wf[N][K] (bf16)
template <int K, int N>
__device__ __forceinline__ void layer_mma(const uint32_t (&a)[K / 16][4], const __nv_bfloat16 *__restrict__ wf,
                                          float (&acc)[N / 8][4], int g, int t) {
#pragma unroll
    for (int nn = 0; nn < N / 8; ++nn) {
        acc[nn][0] = acc[nn][1] = acc[nn][2] = acc[nn][3] = 0.0f;
        const uint32_t *wr = reinterpret_cast<const uint32_t *>(wf + (size_t)(8 * nn + g) * K);
#pragma unroll
        for (int kk = 0; kk < K / 16; ++kk) {
            const uint32_t b0 = __ldg(wr + 8 * kk + t);       // k = 16 kk + 2t, +1
            const uint32_t b1 = __ldg(wr + 8 * kk + 4 + t);   // k = 16 kk + 8 + 2t, +1
            mma_bf16(acc[nn], a[kk], b0, b1);
        }
    }
}

template <int N>
__device__ __forceinline__ void add_bias(float (&acc)[N / 8][4], const float *__restrict__ bias, int t) {
#pragma unroll
    for (int nn = 0; nn < N / 8; ++nn) {
        const float b0 = __ldg(bias + 8 * nn + 2 * t), b1 = __ldg(bias + 8 * nn + 2 * t + 1);
        acc[nn][0] += b0;
        acc[nn][1] += b1;
        acc[nn][2] += b0;
        acc[nn][3] += b1;
    }
}

// input A fragments of a 16-row tile of X [rows][IN] (FP32 in memory, rounded to bf16)
__device__ __forceinline__ void load_input(const float *__restrict__ X, int row0, int nrows, int g, int t,
                                           uint32_t (&a)[IN / 16][4]) {
    const int r0 = row0 + g, r1 = row0 + g + 8;
#pragma unroll
    for (int kk = 0; kk < IN / 16; ++kk) {
        const int c = 16 * kk + 2 * t;
        float2 v00 = make_float2(0.f, 0.f), v10 = v00, v01 = v00, v11 = v00;
        if (r0 < nrows) {
            v00 = *reinterpret_cast<const float2 *>(X + (size_t)r0 * IN + c);
            v01 = *reinterpret_cast<const float2 *>(X + (size_t)r0 * IN + c + 8);
        }
        if (r1 < nrows) {
            v10 = *reinterpret_cast<const float2 *>(X + (size_t)r1 * IN + c);
            v11 = *reinterpret_cast<const float2 *>(X + (size_t)r1 * IN + c + 8);
        }
        a[kk][0] = pack_bf16(v00.x, v00.y);
        a[kk][1] = pack_bf16(v10.x, v10.y);
        a[kk][2] = pack_bf16(v01.x, v01.y);
        a[kk][3] = pack_bf16(v11.x, v11.y);
    }
}

// store accumulator fragments [16 rows x N] as FP32 rows (stride ld)
template <int N>
__device__ __forceinline__ void store_acc(float *__restrict__ Y, int ld, int row0, int nrows, int g, int t,
                                          const float (&acc)[N / 8][4]) {
    const int r0 = row0 + g, r1 = row0 + g + 8;
#pragma unroll
    for (int nn = 0; nn < N / 8; ++nn) {
        const int c = 8 * nn + 2 * t;
        if (r0 < nrows) *reinterpret_cast<float2 *>(Y + (size_t)r0 * ld + c) = make_float2(acc[nn][0], acc[nn][1]);
        if (r1 < nrows) *reinterpret_cast<float2 *>(Y + (size_t)r1 * ld + c) = make_float2(acc[nn][2], acc[nn][3]);
    }
}

// bf16 A-fragment tile [16 rows x K] as rows (stride K)
template <int K>
__device__ __forceinline__ void store_a(__nv_bfloat16 *__restrict__ H, int row0, int nrows, int g, int t,
                                        const uint32_t (&a)[K / 16][4]) {
    const int r0 = row0 + g, r1 = row0 + g + 8;
    uint32_t *h = reinterpret_cast<uint32_t *>(H);
#pragma unroll
    for (int kk = 0; kk < K / 16; ++kk) {
        const int c = 16 * kk + 2 * t;
        if (r0 < nrows) {
            h[((size_t)r0 * K + c) / 2] = a[kk][0];
            h[((size_t)r0 * K + c + 8) / 2] = a[kk][2];
        }
        if (r1 < nrows) {
            h[((size_t)r1 * K + c) / 2] = a[kk][1];
            h[((size_t)r1 * K + c + 8) / 2] = a[kk][3];
        }
    }
}

template <int K>
__device__ __forceinline__ void load_a(const __nv_bfloat16 *__restrict__ H, int row0, int nrows, int g, int t,
                                       uint32_t (&a)[K / 16][4]) {
    const int r0 = row0 + g, r1 = row0 + g + 8;
    const uint32_t *h = reinterpret_cast<const uint32_t *>(H);
#pragma unroll
    for (int kk = 0; kk < K / 16; ++kk) {
        const int c = 16 * kk + 2 * t;
        a[kk][0] = r0 < nrows ? h[((size_t)r0 * K + c) / 2] : 0u;
        a[kk][2] = r0 < nrows ? h[((size_t)r0 * K + c + 8) / 2] : 0u;
        a[kk][1] = r1 < nrows ? h[((size_t)r1 * K + c) / 2] : 0u;
        a[kk][3] = r1 < nrows ? h[((size_t)r1 * K + c + 8) / 2] : 0u;
    }
}

// ---------------------------------------------------------------------------------------------
// forward: Y = MLP(X); with save != 0 also H_l (bf16 layer inputs) and Z_l (FP32 hidden
// pre-activations) for the backward pass.  One warp per 16-sample tile, grid-stride over tiles.
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(32 * WARPS) mlp_forward_kernel(const float *__restrict__ X, int nrows,
                                                                  MlpWeights w, float *__restrict__ Y,
                                                                  __nv_bfloat16 *__restrict__ H0,
                                                                  __nv_bfloat16 *__restrict__ Hh,
                                                                  float *__restrict__ Z) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int ntile = (nrows + 15) / 16;
    for (int tile = blockIdx.x * WARPS + (threadIdx.x >> 5); tile < ntile; tile += gridDim.x * WARPS) {
        const int row0 = tile * 16;
        uint32_t a0[IN / 16][4];
        load_input(X, row0, nrows, g, t, a0);
        if (H0) store_a<IN>(H0, row0, nrows, g, t, a0);
        float acc[HID / 8][4];
        layer_mma<IN, HID>(a0, w.wf[0], acc, g, t);
        add_bias<HID>(acc, w.bias[0], t);
        uint32_t ah[HID / 16][4];
#pragma unroll
        for (int l = 1; l < NL; ++l) {
            if (Z) store_acc<HID>(Z + (size_t)(l - 1) * nrows * HID, HID, row0, nrows, g, t, acc);
#pragma unroll
            for (int nn = 0; nn < HID / 8; ++nn)
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[nn][q] = gelu(acc[nn][q]);
            acc_to_a<HID>(acc, ah);
            if (Hh) store_a<HID>(Hh + (size_t)(l - 1) * nrows * HID, row0, nrows, g, t, ah);
            if (l < NL - 1) {
                layer_mma<HID, HID>(ah, w.wf[l], acc, g, t);
                add_bias<HID>(acc, w.bias[l], t);
            }
        }
        float out[OUT / 8][4];
        layer_mma<HID, OUT>(ah, w.wf[NL - 1], out, g, t);
        add_bias<OUT>(out, w.bias[NL - 1], t);
        store_acc<OUT>(Y, OUT, row0, nrows, g, t, out);
    }
}

// ---------------------------------------------------------------------------------------------
// backward of the mean-squared loss over the first nout outputs:
//   L = sum_rows sum_{c < nout} (Y - T)^2 / (nrows nout)
// One CTA per 64-sample block: dZ fragments flow back through the layers in registers
// (dH = dZ W^T, dZ = dH * GELU'(Z)); the weight gradient of each layer, H^T dZ over the block's
// samples, is formed from shared-memory copies of H and dZ and written as the block's partial
// (reduced across blocks by mlp_reduce_kernel).
// ---------------------------------------------------------------------------------------------
constexpr int GW_ELEMS = IN * HID + 2 * HID * HID + HID * OUT;   // weight elements
constexpr int GB_ELEMS = 3 * HID + OUT;                          // bias elements
__host__ __device__ constexpr int w_off(int l) { return l == 0 ? 0 : IN * HID + (l - 1) * HID * HID; }
__host__ __device__ constexpr int b_off(int l) { return l * HID; }

template <int K, int N>
__device__ void block_wgrad(const __nv_bfloat16 *sH, const __nv_bfloat16 *sD, float *gw, float *gb) {
    // gw[k][n] = sum_r sH[r][k] sD[r][n] over ROWS samples; warp w takes n tiles w, w + 4, ...
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3, w = threadIdx.x >> 5;
    for (int nn = w; nn < N / 8; nn += WARPS) {
        for (int mm = 0; mm < K / 16; ++mm) {
            float d[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int kk = 0; kk < ROWS / 16; ++kk) {
                // A = H^T (16 k-rows of weight index x 16 samples), B = dZ (16 samples x 8 outputs)
                const int r = 16 * kk + 2 * t;
                const int m0 = 16 * mm + g, m1 = m0 + 8;
                uint32_t a[4];
                a[0] = pack_bf16(__bfloat162float(sH[r * K + m0]), __bfloat162float(sH[(r + 1) * K + m0]));
                a[1] = pack_bf16(__bfloat162float(sH[r * K + m1]), __bfloat162float(sH[(r + 1) * K + m1]));
                a[2] = pack_bf16(__bfloat162float(sH[(r + 8) * K + m0]), __bfloat162float(sH[(r + 9) * K + m0]));
                a[3] = pack_bf16(__bfloat162float(sH[(r + 8) * K + m1]), __bfloat162float(sH[(r + 9) * K + m1]));
                const int n = 8 * nn + g;
                const uint32_t b0 = pack_bf16(__bfloat162float(sD[r * N + n]), __bfloat162float(sD[(r + 1) * N + n]));
                const uint32_t b1 = pack_bf16(__bfloat162float(sD[(r + 8) * N + n]), __bfloat162float(sD[(r + 9) * N + n]));
                mma_bf16(d, a, b0, b1);
            }
            const int m0 = 16 * mm + g, c = 8 * nn + 2 * t;
            gw[(size_t)m0 * N + c] = d[0];
            gw[(size_t)m0 * N + c + 1] = d[1];
            gw[(size_t)(m0 + 8) * N + c] = d[2];
            gw[(size_t)(m0 + 8) * N + c + 1] = d[3];
        }
    }
    // bias gradient: column sums of dZ (FP32 from the bf16 copy)
    for (int n = threadIdx.x; n < N; n += blockDim.x) {
        float s = 0.f;
        for (int r = 0; r < ROWS; ++r) s += __bfloat162float(sD[r * N + n]);
        gb[n] = s;
    }
}

__global__ void __launch_bounds__(32 * WARPS) mlp_backward_kernel(const float *__restrict__ Y,
                                                                   const float *__restrict__ T, int nrows,
                                                                   int nout, MlpWeights w,
                                                                   const __nv_bfloat16 *__restrict__ H0,
                                                                   const __nv_bfloat16 *__restrict__ Hh,
                                                                   const float *__restrict__ Z,
                                                                   float *__restrict__ gw_part,
                                                                   float *__restrict__ gb_part) {
    __shared__ __align__(16) __nv_bfloat16 sH[ROWS * HID];
    __shared__ __align__(16) __nv_bfloat16 sD[ROWS * HID];
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3, wp = threadIdx.x >> 5;
    const int row0 = blockIdx.x * ROWS + 16 * wp;
    const int r0 = row0 + g, r1 = row0 + g + 8;
    float *gw = gw_part + (size_t)blockIdx.x * GW_ELEMS;
    float *gb = gb_part + (size_t)blockIdx.x * GB_ELEMS;
    const float scale = 2.0f / ((float)nrows * (float)nout);
    // dZ of the output layer (linear): dL/dY
    float dz[OUT / 8][4];
#pragma unroll
    for (int nn = 0; nn < OUT / 8; ++nn)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int r = (q < 2) ? r0 : r1, c = 8 * nn + 2 * t + (q & 1);
            float v = 0.f;
            if (r < nrows && c < nout) v = scale * (Y[(size_t)r * OUT + c] - T[(size_t)r * nout + c]);
            dz[nn][q] = v;
        }
    uint32_t adz[OUT / 16][4];
    acc_to_a<OUT>(dz, adz);
    // ---- layer NL-1 (HID -> OUT) ----
    {
        uint32_t ah[HID / 16][4];
        load_a<HID>(Hh + (size_t)(NL - 2) * nrows * HID, row0, nrows, g, t, ah);
        store_a<HID>(sH, 16 * wp, ROWS, g, t, ah);
        store_a<OUT>(sD, 16 * wp, ROWS, g, t, adz);
        __syncthreads();
        block_wgrad<HID, OUT>(sH, sD, gw + w_off(NL - 1), gb + b_off(NL - 1));
        __syncthreads();
    }
    // dH = dZ W^T: W^T given by wb[in][out] rows (in = output index n of this product)
    float dh[HID / 8][4];
    layer_mma<OUT, HID>(adz, w.wb[NL - 1], dh, g, t);
    for (int l = NL - 2; l >= 0; --l) {
        // dZ_l = dH * GELU'(Z_l)
        const float *Zl = Z + (size_t)l * nrows * HID;
#pragma unroll
        for (int nn = 0; nn < HID / 8; ++nn)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int r = (q < 2) ? r0 : r1, c = 8 * nn + 2 * t + (q & 1);
                dh[nn][q] = (r < nrows) ? dh[nn][q] * gelu_d(Zl[(size_t)r * HID + c]) : 0.f;
            }
        uint32_t ad[HID / 16][4];
        acc_to_a<HID>(dh, ad);
        const int K = layer_in(l);
        if (l == 0) {
            uint32_t ah[IN / 16][4];
            load_a<IN>(H0, row0, nrows, g, t, ah);
            store_a<IN>(sH, 16 * wp, ROWS, g, t, ah);
        } else {
            uint32_t ah[HID / 16][4];
            load_a<HID>(Hh + (size_t)(l - 1) * nrows * HID, row0, nrows, g, t, ah);
            store_a<HID>(sH, 16 * wp, ROWS, g, t, ah);
        }
        store_a<HID>(sD, 16 * wp, ROWS, g, t, ad);
        __syncthreads();
        if (K == IN)
            block_wgrad<IN, HID>(sH, sD, gw + w_off(l), gb + b_off(l));
        else
            block_wgrad<HID, HID>(sH, sD, gw + w_off(l), gb + b_off(l));
        __syncthreads();
        if (l > 0) layer_mma<HID, HID>(ad, w.wb[l], dh, g, t);
    }
}

// sum the per-block partial gradients (fixed order: deterministic)
__global__ void mlp_reduce_kernel(const float *__restrict__ part, int nblocks, int n, float *__restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float s = 0.f;
        for (int b = 0; b < nblocks; ++b) s += part[(size_t)b * n + i];
        out[i] = s;
    }
}

// Adam on the FP32 master weights [in][out] and biases; refresh both bf16 layouts
__global__ void mlp_adam_kernel(float *__restrict__ master_w, float *__restrict__ master_b,
                                const float *__restrict__ gw, const float *__restrict__ gb,
                                float *__restrict__ mw, float *__restrict__ vw, float *__restrict__ mb,
                                float *__restrict__ vb, __nv_bfloat16 *__restrict__ wf,
                                __nv_bfloat16 *__restrict__ wb, float lr, float b1, float b2, float eps,
                                float bc1, float bc2, float wd) {
    const int nw = GW_ELEMS, nb = GB_ELEMS;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nw + nb; i += gridDim.x * blockDim.x) {
        if (i < nw) {
            const float gr = gw[i];
            const float m = b1 * mw[i] + (1.f - b1) * gr;
            const float v = b2 * vw[i] + (1.f - b2) * gr * gr;
            mw[i] = m;
            vw[i] = v;
            float p = master_w[i];
            p -= lr * ((m / bc1) / (sqrtf(v / bc2) + eps) + wd * p);
            master_w[i] = p;
            // layer and position of element i ([in][out] within the layer)
            int l = 0;
            while (l < NL - 1 && i >= w_off(l + 1)) ++l;
            const int K = layer_in(l), N = layer_out(l);
            const int j = i - w_off(l), k = j / N, n = j - (j / N) * N;
            const __nv_bfloat16 h = __float2bfloat16_rn(p);
            wb[w_off(l) + k * N + n] = h;
            wf[w_off(l) + n * K + k] = h;
        } else {
            const int j = i - nw;
            const float gr = gb[j];
            const float m = b1 * mb[j] + (1.f - b1) * gr;
            const float v = b2 * vb[j] + (1.f - b2) * gr * gr;
            mb[j] = m;
            vb[j] = v;
            master_b[j] -= lr * (m / bc1) / (sqrtf(v / bc2) + eps);
        }
    }
}

// ---------------------------------------------------------------------------------------------
// closure features and correction (coarse grid, order CN = 6)
//   sample (e, i, a, b): x node i of interior x element e, interior velocity element (a, b)
//   features: the element's 6 x 6 nodal patch f[e, i, a, :, b, :], the neighbour traces of the
//   four adjacent velocity elements (their first and second node lines next to the shared face),
//   each divided by the sample's scale max|.|; then a E_i / escale, the element's centre u / umax
//   and v / vmax, and a B; zero padding to IN.
// ---------------------------------------------------------------------------------------------
constexpr int CN = 6;
constexpr int NF = CN * CN + 8 * CN;   // 84 state values

template <typename T>
__global__ void closure_features_kernel(const T *__restrict__ f, int nx, int nu, int nv,
                                        const double *__restrict__ E, double accel, double bfield,
                                        const double *__restrict__ un, const double *__restrict__ vn,
                                        double umax, double vmax, double escale, float *__restrict__ X,
                                        float *__restrict__ scale) {
    const int U = nu + 2, V = nv + 2;
    const long sJ = (long)V * CN, sA = sJ * CN, sI = sA * U, sE = sI * CN;
    const long total = (long)nx * CN * nu * nv;
    for (long s = blockIdx.x * (long)blockDim.x + threadIdx.x; s < total; s += (long)gridDim.x * blockDim.x) {
        long r = s;
        const int b = (int)(r % nv) + 1; r /= nv;
        const int a = (int)(r % nu) + 1; r /= nu;
        const int i = (int)(r % CN); r /= CN;
        const int e = (int)r + 1;
        const T *p = f + e * sE + i * sI;
        float v[NF];
        int q = 0;
        for (int j = 0; j < CN; ++j)
            for (int k = 0; k < CN; ++k) v[q++] = (float)p[a * sA + j * sJ + b * CN + k];
        for (int k = 0; k < CN; ++k) v[q++] = (float)p[(a - 1) * sA + (CN - 1) * sJ + b * CN + k];
        for (int k = 0; k < CN; ++k) v[q++] = (float)p[(a + 1) * sA + 0 * sJ + b * CN + k];
        for (int j = 0; j < CN; ++j) v[q++] = (float)p[a * sA + j * sJ + (b - 1) * CN + CN - 1];
        for (int j = 0; j < CN; ++j) v[q++] = (float)p[a * sA + j * sJ + (b + 1) * CN + 0];
        for (int k = 0; k < CN; ++k) v[q++] = (float)p[(a - 1) * sA + (CN - 2) * sJ + b * CN + k];
        for (int k = 0; k < CN; ++k) v[q++] = (float)p[(a + 1) * sA + 1 * sJ + b * CN + k];
        for (int j = 0; j < CN; ++j) v[q++] = (float)p[a * sA + j * sJ + (b - 1) * CN + CN - 2];
        for (int j = 0; j < CN; ++j) v[q++] = (float)p[a * sA + j * sJ + (b + 1) * CN + 1];
        float m = 0.f;
        for (int c = 0; c < NF; ++c) m = fmaxf(m, fabsf(v[c]));
        m = fmaxf(m, 1e-30f);
        float *x = X + s * IN;
        for (int c = 0; c < NF; ++c) x[c] = v[c] / m;
        x[NF + 0] = (float)(accel * E[e * CN + i] / escale);
        x[NF + 1] = (float)(0.5 * (un[a * CN] + un[a * CN + CN - 1]) / umax);
        x[NF + 2] = (float)(0.5 * (vn[b * CN] + vn[b * CN + CN - 1]) / vmax);
        x[NF + 3] = (float)(accel * bfield);
        for (int c = NF + 4; c < IN; ++c) x[c] = 0.f;
        scale[s] = m;
    }
}

// out[e, i, a, j, b, k] += c2 dt cscale scale[s] clamp(Y[s][j CN + k], +-ymax)
template <typename T>
__global__ void closure_apply_kernel(T *__restrict__ out, int nx, int nu, int nv, const float *__restrict__ Y,
                                     const float *__restrict__ scale, double cscale, float ymax,
                                     const double *__restrict__ dt, double c2,
                                     const vl_run_state *__restrict__ state) {
    if (state != nullptr && state->active == 0) return;
    const int U = nu + 2, V = nv + 2;
    const long sJ = (long)V * CN, sA = sJ * CN, sI = sA * U, sE = sI * CN;
    const long total = (long)nx * CN * nu * nv * CN * CN;
    const double w = c2 * (*dt) * cscale;
    for (long p = blockIdx.x * (long)blockDim.x + threadIdx.x; p < total; p += (long)gridDim.x * blockDim.x) {
        long r = p;
        const int k = (int)(r % CN); r /= CN;
        const int j = (int)(r % CN); r /= CN;
        const long s = r;
        const int b = (int)(r % nv) + 1; r /= nv;
        const int a = (int)(r % nu) + 1; r /= nu;
        const int i = (int)(r % CN); r /= CN;
        const int e = (int)r + 1;
        const long o = e * sE + i * sI + a * sA + j * sJ + b * CN + k;
        const float y = fminf(fmaxf(Y[s * OUT + j * CN + k], -ymax), ymax);
        out[o] = (T)((double)out[o] + w * (double)scale[s] * (double)y);
    }
}

// Charge-conserving form: one CTA per x node (e, i) removes from the correction of that node the
// quadrature mean over all of its velocity nodes, so the correction leaves the zeroth moment -- the
// charge density the field is solved from -- unchanged:
//   c[s, j, k] = scale[s] clamp(Y[s][6 j + k]),  mean = sum w_j w_k c / sum w_j w_k,
//   out += c2 dt cscale (c - mean)
struct NodeWeights {
    double w[CN];
};

constexpr int CONS_THREADS = 256;

template <typename T>
__global__ void __launch_bounds__(CONS_THREADS)
closure_apply_conservative_kernel(T *__restrict__ out, int nx, int nu, int nv, const float *__restrict__ Y,
                                  const float *__restrict__ scale, double cscale, float ymax,
                                  const double *__restrict__ dt, double c2, const vl_run_state *__restrict__ state,
                                  const NodeWeights wq) {
    __shared__ double s_part[CONS_THREADS / 32];
    if (state != nullptr && state->active == 0) return;
    const int node = blockIdx.x;   // e CN + i, e 0-based
    const int e = node / CN + 1, i = node % CN;
    const int U = nu + 2, V = nv + 2;
    const long sJ = (long)V * CN, sA = sJ * CN, sI = sA * U, sE = sI * CN;
    const long nsamp = (long)nu * nv;
    const long s0 = (long)node * nsamp;
    const long count = nsamp * CN * CN;
    double acc = 0.0;
    for (long q = threadIdx.x; q < count; q += blockDim.x) {
        const long s = s0 + q / (CN * CN);
        const int jk = (int)(q % (CN * CN));
        const float y = fminf(fmaxf(Y[s * OUT + jk], -ymax), ymax);
        acc = fma(wq.w[jk / CN] * wq.w[jk % CN], (double)scale[s] * (double)y, acc);
    }
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = acc;
    __syncthreads();
    double tot = 0.0, wsum = 0.0;
    for (int w = 0; w < CONS_THREADS / 32; ++w) tot += s_part[w];
    for (int j = 0; j < CN; ++j)
        for (int k = 0; k < CN; ++k) wsum += wq.w[j] * wq.w[k];
    const double mean = tot / (wsum * (double)nsamp);
    const double w = c2 * (*dt) * cscale;
    for (long q = threadIdx.x; q < count; q += blockDim.x) {
        const long s = s0 + q / (CN * CN);
        const int jk = (int)(q % (CN * CN));
        const int j = jk / CN, k = jk % CN;
        const long sl = s - s0;
        const int a = (int)(sl / nv) + 1, b = (int)(sl % nv) + 1;
        const long o = e * sE + i * sI + a * sA + j * sJ + b * CN + k;
        const float y = fminf(fmaxf(Y[s * OUT + jk], -ymax), ymax);
        out[o] = (T)((double)out[o] + w * ((double)scale[s] * (double)y - mean));
    }
}

MlpWeights weights_of(const __nv_bfloat16 *wf, const __nv_bfloat16 *wb, const float *bias) {
    MlpWeights w;
    for (int l = 0; l < NL; ++l) {
        w.wf[l] = wf + w_off(l);
        w.wb[l] = wb + w_off(l);
        w.bias[l] = bias + b_off(l);
    }
    return w;
}

int fail(int code, const char *msg) {
    vl_internal_set_error(msg);
    return code;
}

int check(const char *where) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        vl_internal_set_error((std::string(where) + ": " + cudaGetErrorString(e)).c_str());
        return VL_ERR_CUDA;
    }
    return VL_OK;
}

}  // namespace

extern "C" {

VL_API int vl_closure_features(const void *f, int32_t prec, int32_t nx, int32_t nu, int32_t nv,
                               const double *E, double accel, double bfield, const double *u_nodes,
                               const double *v_nodes, double umax, double vmax, double escale, float *X,
                               float *scale, void *stream) {
    if (!f || !E || !u_nodes || !v_nodes || !X || !scale) return fail(VL_ERR_INVALID, "null argument");
    if (nx < 1 || nu < 1 || nv < 1) return fail(VL_ERR_INVALID, "empty grid");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const long total = (long)nx * CN * nu * nv;
    const int blocks = (int)((total + 127) / 128 < 148 * 32 ? (total + 127) / 128 : 148 * 32);
    if (prec == VL_FP64)
        closure_features_kernel<double><<<blocks, 128, 0, s>>>(static_cast<const double *>(f), nx, nu, nv, E, accel,
                                                               bfield, u_nodes, v_nodes, umax, vmax, escale, X, scale);
    else
        closure_features_kernel<float><<<blocks, 128, 0, s>>>(static_cast<const float *>(f), nx, nu, nv, E, accel,
                                                              bfield, u_nodes, v_nodes, umax, vmax, escale, X, scale);
    return check("closure_features_kernel");
}

VL_API int vl_closure_apply(void *out, int32_t prec, int32_t nx, int32_t nu, int32_t nv, const float *Y,
                            const float *scale, double cscale, float ymax, const double *dt, double c2,
                            const vl_run_state *state, int32_t mode, const double *node_weights, void *stream) {
    if (!out || !Y || !scale || !dt) return fail(VL_ERR_INVALID, "null argument");
    if (mode != VL_CLOSURE_PLAIN && mode != VL_CLOSURE_CHARGE) return fail(VL_ERR_INVALID, "closure mode");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (mode == VL_CLOSURE_CHARGE) {
        if (!node_weights) return fail(VL_ERR_INVALID, "null node weights");
        NodeWeights wq;
        for (int j = 0; j < CN; ++j) wq.w[j] = node_weights[j];
        const int blocks = nx * CN;
        if (prec == VL_FP64)
            closure_apply_conservative_kernel<double><<<blocks, CONS_THREADS, 0, s>>>(
                static_cast<double *>(out), nx, nu, nv, Y, scale, cscale, ymax, dt, c2, state, wq);
        else
            closure_apply_conservative_kernel<float><<<blocks, CONS_THREADS, 0, s>>>(
                static_cast<float *>(out), nx, nu, nv, Y, scale, cscale, ymax, dt, c2, state, wq);
        return check("closure_apply_conservative_kernel");
    }
    const long total = (long)nx * CN * nu * nv * CN * CN;
    const int blocks = (int)((total + 255) / 256 < 148 * 32 ? (total + 255) / 256 : 148 * 32);
    if (prec == VL_FP64)
        closure_apply_kernel<double><<<blocks, 256, 0, s>>>(static_cast<double *>(out), nx, nu, nv, Y, scale,
                                                            cscale, ymax, dt, c2, state);
    else
        closure_apply_kernel<float><<<blocks, 256, 0, s>>>(static_cast<float *>(out), nx, nu, nv, Y, scale,
                                                           cscale, ymax, dt, c2, state);
    return check("closure_apply_kernel");
}

VL_API int vl_mlp_dims(int32_t *in, int32_t *hidden, int32_t *out, int32_t *n_weights, int32_t *n_bias) {
    if (in) *in = IN;
    if (hidden) *hidden = HID;
    if (out) *out = OUT;
    if (n_weights) *n_weights = GW_ELEMS;
    if (n_bias) *n_bias = GB_ELEMS;
    return VL_OK;
}

VL_API int vl_mlp_forward(const float *X, int32_t nrows, const void *wf, const void *wb, const float *bias,
                          float *Y, void *H0, void *Hh, float *Z, void *stream) {
    if (!X || !wf || !wb || !bias || !Y || nrows < 0) return fail(VL_ERR_INVALID, "null argument");
    if (nrows == 0) return VL_OK;
    const bool save = H0 || Hh || Z;
    if (save && !(H0 && Hh && Z)) return fail(VL_ERR_INVALID, "training forward needs H0, Hh and Z");
    const int tiles = (nrows + 15) / 16;
    int blocks = (tiles + WARPS - 1) / WARPS;
    if (blocks > 148 * 16) blocks = 148 * 16;
    mlp_forward_kernel<<<blocks, 32 * WARPS, 0, static_cast<cudaStream_t>(stream)>>>(
        X, nrows, weights_of(static_cast<const __nv_bfloat16 *>(wf), static_cast<const __nv_bfloat16 *>(wb), bias),
        Y, static_cast<__nv_bfloat16 *>(H0), static_cast<__nv_bfloat16 *>(Hh), Z);
    return check("mlp_forward_kernel");
}

VL_API size_t vl_mlp_partial_floats(int32_t nrows) {
    const size_t blocks = (size_t)(nrows + ROWS - 1) / ROWS;
    return blocks * (GW_ELEMS + GB_ELEMS);
}

VL_API int vl_mlp_backward(const float *Y, const float *T, int32_t nrows, int32_t nout, const void *wf,
                           const void *wb, const float *bias, const void *H0, const void *Hh, const float *Z,
                           float *partials, float *grad_w, float *grad_b, void *stream) {
    if (!Y || !T || !wf || !wb || !bias || !H0 || !Hh || !Z || !partials || !grad_w || !grad_b)
        return fail(VL_ERR_INVALID, "null argument");
    if (nrows < 1 || nout < 1 || nout > OUT) return fail(VL_ERR_INVALID, "nrows >= 1, nout in 1..48");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int blocks = (nrows + ROWS - 1) / ROWS;
    float *gw_part = partials;
    float *gb_part = partials + (size_t)blocks * GW_ELEMS;
    mlp_backward_kernel<<<blocks, 32 * WARPS, 0, s>>>(
        Y, T, nrows, nout,
        weights_of(static_cast<const __nv_bfloat16 *>(wf), static_cast<const __nv_bfloat16 *>(wb), bias),
        static_cast<const __nv_bfloat16 *>(H0), static_cast<const __nv_bfloat16 *>(Hh), Z, gw_part, gb_part);
    int rc = check("mlp_backward_kernel");
    if (rc) return rc;
    mlp_reduce_kernel<<<148 * 4, 256, 0, s>>>(gw_part, blocks, GW_ELEMS, grad_w);
    if ((rc = check("mlp_reduce_kernel(w)"))) return rc;
    mlp_reduce_kernel<<<4, 128, 0, s>>>(gb_part, blocks, GB_ELEMS, grad_b);
    return check("mlp_reduce_kernel(b)");
}

VL_API int vl_mlp_adam(float *master_w, float *master_b, const float *grad_w, const float *grad_b, float *m_w,
                       float *v_w, float *m_b, float *v_b, void *wf, void *wb, float lr, float beta1,
                       float beta2, float eps, int32_t step, float weight_decay, void *stream) {
    if (!master_w || !master_b || !grad_w || !grad_b || !m_w || !v_w || !m_b || !v_b || !wf || !wb || step < 1)
        return fail(VL_ERR_INVALID, "null argument or step < 1");
    float bc1 = 1.f, bc2 = 1.f;
    for (int i = 0; i < step && i < 100000; ++i) {
        bc1 *= beta1;
        bc2 *= beta2;
    }
    bc1 = 1.f - bc1;
    bc2 = 1.f - bc2;
    mlp_adam_kernel<<<148 * 2, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        master_w, master_b, grad_w, grad_b, m_w, v_w, m_b, v_b, static_cast<__nv_bfloat16 *>(wf),
        static_cast<__nv_bfloat16 *>(wb), lr, beta1, beta2, eps, bc1, bc2, weight_decay);
    return check("mlp_adam_kernel");
}

}  // extern "C"
