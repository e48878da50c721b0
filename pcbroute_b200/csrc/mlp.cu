// The conflict predictor's network: a 3-layer MLP (D0 -> 128 -> 128 -> 1) with BF16 operands and FP32
// accumulation, trained and evaluated by the kernels below.
//
//   z1 = x W1^T + b1, h1 = relu(z1)        x [B][D0] bf16, W1 [128][D0] bf16
//   z2 = h1 W2^T + b2, h2 = relu(z2)       h1 stored bf16, W2 [128][128] bf16
//   z3 = h2 . w3 + b3, p = sigmoid(z3)     loss: mean binary cross-entropy over the valid rows
//
// Every product runs through one tensor-core GEMM, C[M][N] = sum_k A[m][k] B[n][k] (both operands K-contiguous),
// built on mma.sync m16n8k16 (bf16 x bf16 -> f32): 64 x 64 tiles, 4 warps of 32 x 32, K staged 32 at a time in
// shared memory. The epilogue adds a bias, applies relu or a relu mask from another tensor, and writes f32, bf16
// and / or transposed bf16, so the backward pass finds every operand K-contiguous:
//   dW2 = dz2^T h1   (A = dz2^T [128][B], B = h1^T [128][B])
//   dh1 = dz2 W2     (A = dz2 [B][128], B = W2^T [128][128])
//   dW1 = dz1^T x    (A = dz1^T [128][B], B = x^T [D0][B])
// The network is small (about 0.3 M parameters); its cost is a rounding error next to the searches it schedules,
// so these kernels aim at exactness and simplicity rather than at the tensor-core roofline.
#include <cuda_bf16.h>

#include <cmath>
#include <vector>

#include "pcbg_internal.h"

namespace pcbg {

namespace {

constexpr int GM = 64, GN = 64, GK = 32, GPAD = 8;

enum Epi : int {
    EPI_BIAS = 1,        // + bias[n]
    EPI_RELU = 2,        // max(0, .)
    EPI_MASK = 4,        // * (mask[m][n] > 0), mask bf16 [M][ldm]
};

__device__ __forceinline__ void mma16816(float (&c)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// C[M][N] = A[M][K] . B[N][K]^T with the epilogue above. M, N multiples of 64, K a multiple of 32; lda / ldb / the
// output strides in elements; every row start 16-byte aligned.
__global__ void __launch_bounds__(128) gemm_tn_kernel(const __nv_bfloat16* A, int lda, const __nv_bfloat16* Bm, int ldb,
                                                      int M, int N, int K, int epi, const float* bias,
                                                      const __nv_bfloat16* mask, int ldm, float* Cf, int ldcf,
                                                      __nv_bfloat16* Cb, int ldcb, __nv_bfloat16* Ct, int ldct) {
    __shared__ __align__(16) __nv_bfloat16 As[GM][GK + GPAD];
    __shared__ __align__(16) __nv_bfloat16 Bs[GN][GK + GPAD];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * GM, n0 = blockIdx.x * GN;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    const int g = lane >> 2, t = lane & 3;
    float acc[2][4][4];
    #pragma unroll
    for (int a = 0; a < 2; ++a)
        #pragma unroll
        for (int b = 0; b < 4; ++b)
            #pragma unroll
            for (int c = 0; c < 4; ++c) acc[a][b][c] = 0.f;
    for (int k0 = 0; k0 < K; k0 += GK) {
        // stage: 64 rows x 32 bf16 = 256 chunks of 16 bytes per operand, 2 per thread
        #pragma unroll
        for (int r = 0; r < 2; ++r) {
            const int ch = tid + r * 128, row = ch >> 2, col = (ch & 3) * 8;
            *reinterpret_cast<uint4*>(&As[row][col]) =
                *reinterpret_cast<const uint4*>(A + size_t(m0 + row) * lda + k0 + col);
            *reinterpret_cast<uint4*>(&Bs[row][col]) =
                *reinterpret_cast<const uint4*>(Bm + size_t(n0 + row) * ldb + k0 + col);
        }
        __syncthreads();
        #pragma unroll
        for (int kk = 0; kk < GK; kk += 16) {
            uint32_t af[2][4], bf[4][2];
            #pragma unroll
            for (int a = 0; a < 2; ++a) {
                const int r = wm + a * 16 + g;
                af[a][0] = *reinterpret_cast<const uint32_t*>(&As[r][kk + 2 * t]);
                af[a][1] = *reinterpret_cast<const uint32_t*>(&As[r + 8][kk + 2 * t]);
                af[a][2] = *reinterpret_cast<const uint32_t*>(&As[r][kk + 2 * t + 8]);
                af[a][3] = *reinterpret_cast<const uint32_t*>(&As[r + 8][kk + 2 * t + 8]);
            }
            #pragma unroll
            for (int b = 0; b < 4; ++b) {
                const int c = wn + b * 8 + g;
                bf[b][0] = *reinterpret_cast<const uint32_t*>(&Bs[c][kk + 2 * t]);
                bf[b][1] = *reinterpret_cast<const uint32_t*>(&Bs[c][kk + 2 * t + 8]);
            }
            #pragma unroll
            for (int a = 0; a < 2; ++a)
                #pragma unroll
                for (int b = 0; b < 4; ++b) mma16816(acc[a][b], af[a], bf[b]);
        }
        __syncthreads();
    }
    #pragma unroll
    for (int a = 0; a < 2; ++a)
        #pragma unroll
        for (int b = 0; b < 4; ++b)
            #pragma unroll
            for (int c = 0; c < 4; ++c) {
                const int m = m0 + wm + a * 16 + g + (c >= 2 ? 8 : 0);
                const int n = n0 + wn + b * 8 + 2 * t + (c & 1);
                float v = acc[a][b][c];
                if (epi & EPI_BIAS) v += bias[n];
                if (epi & EPI_RELU) v = fmaxf(v, 0.f);
                if (epi & EPI_MASK) v = __bfloat162float(mask[size_t(m) * ldm + n]) > 0.f ? v : 0.f;
                if (Cf) Cf[size_t(m) * ldcf + n] = v;
                const __nv_bfloat16 h = __float2bfloat16_rn(v);
                if (Cb) Cb[size_t(m) * ldcb + n] = h;
                if (Ct) Ct[size_t(n) * ldct + m] = h;
            }
}

// head: z3 = h2 . w3 + b3 per row (one warp per row), p = sigmoid(z3)
__global__ void head_forward_kernel(const __nv_bfloat16* h2, const float* w3, const float* b3, int B, float* z, float* p) {
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (row >= B) return;
    float s = 0.f;
    for (int j = lane; j < MLP_H; j += 32) s += __bfloat162float(h2[size_t(row) * MLP_H + j]) * w3[j];
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
    if (lane == 0) {
        const float v = s + b3[0];
        z[row] = v;
        if (p) p[row] = 1.f / (1.f + expf(-v));
    }
}

// head backward + loss: dz3 = (sigmoid(z3) - y) * w / sum(w); dw3 += dz3 h2; db3 += dz3;
// dz2 = dz3 w3 * (h2 > 0), written bf16 [B][H] and transposed [H][B]. Rows with weight 0 (padding) give 0.
__global__ void head_backward_kernel(const __nv_bfloat16* h2, const float* z, const float* y, const float* w, float wsum,
                                     const float* w3, int B, float* dw3, float* db3, __nv_bfloat16* dz2,
                                     __nv_bfloat16* dz2t, float* loss) {
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (row >= B) return;
    const float zz = z[row], ww = w[row];
    const float sg = 1.f / (1.f + expf(-zz));
    const float d = ww > 0.f ? (sg - y[row]) * ww / wsum : 0.f;
    if (lane == 0 && ww > 0.f) {
        // BCE with logits: max(z, 0) - z y + log(1 + exp(-|z|))
        const float l = fmaxf(zz, 0.f) - zz * y[row] + log1pf(expf(-fabsf(zz)));
        atomicAdd(loss, l * ww / wsum);
        atomicAdd(db3, d);
    }
    for (int j = lane; j < MLP_H; j += 32) {
        const float hv = __bfloat162float(h2[size_t(row) * MLP_H + j]);
        if (d != 0.f) atomicAdd(&dw3[j], d * hv);
        const __nv_bfloat16 g = __float2bfloat16_rn(hv > 0.f ? d * w3[j] : 0.f);
        dz2[size_t(row) * MLP_H + j] = g;
        dz2t[size_t(j) * B + row] = g;
    }
}

// column sums: db[n] = sum_m d[m][n] (bf16 d, f32 sums)
__global__ void colsum_kernel(const __nv_bfloat16* d, int M, int N, float* out) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    float s = 0.f;
    for (int m = 0; m < M; ++m) s += __bfloat162float(d[size_t(m) * N + n]);
    out[n] = s;
}

// x [R][C] bf16 -> xt [C][R]
__global__ void transpose_bf16_kernel(const __nv_bfloat16* x, int R, int C, __nv_bfloat16* xt) {
    __shared__ __nv_bfloat16 t[32][33];
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int r = r0 + k, c = c0 + threadIdx.x;
        if (r < R && c < C) t[k][threadIdx.x] = x[size_t(r) * C + c];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int c = c0 + k, r = r0 + threadIdx.x;
        if (r < R && c < C) xt[size_t(c) * R + r] = t[threadIdx.x][k];
    }
}

// Adam on f32 master weights, then the bf16 copy (and, for W2, its transpose: ldt > 0, rows x cols = H x H)
__global__ void adam_kernel(float* wgt, const float* grad, float* m, float* v, int n, float lr, float b1, float b2,
                            float eps, float c1, float c2, __nv_bfloat16* wb, __nv_bfloat16* wt, int cols) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const float gk = grad[k];
        const float mk = b1 * m[k] + (1.f - b1) * gk;
        const float vk = b2 * v[k] + (1.f - b2) * gk * gk;
        m[k] = mk;
        v[k] = vk;
        const float w = wgt[k] - lr * (mk / c1) / (sqrtf(vk / c2) + eps);
        wgt[k] = w;
        if (wb) wb[k] = __float2bfloat16_rn(w);
        if (wt) wt[size_t(k % cols) * (n / cols) + k / cols] = __float2bfloat16_rn(w);
    }
}

__global__ void cast_bf16_kernel(const float* x, int n, __nv_bfloat16* y, __nv_bfloat16* yt, int cols) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        y[k] = __float2bfloat16_rn(x[k]);
        if (yt) yt[size_t(k % cols) * (n / cols) + k / cols] = __float2bfloat16_rn(x[k]);
    }
}

int gemm(cudaStream_t s, const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb, int M, int N, int K, int epi,
         const float* bias, const __nv_bfloat16* mask, int ldm, float* Cf, int ldcf, __nv_bfloat16* Cb, int ldcb,
         __nv_bfloat16* Ct, int ldct) {
    if (M % GM || N % GN || K % GK || lda % 8 || ldb % 8) {
        set_error("gemm shape not a multiple of the tile");
        return -1;
    }
    gemm_tn_kernel<<<dim3(N / GN, M / GM), 128, 0, s>>>(A, lda, B, ldb, M, N, K, epi, bias, mask, ldm, Cf, ldcf, Cb, ldcb, Ct, ldct);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace

// ---- the network object ----

Mlp::~Mlp() {
    for (void* p : owned) cudaFree(p);
}

bool Mlp::init(uint64_t seed) {
    auto alloc = [&](size_t bytes) -> void* {
        void* p = nullptr;
        if (cudaMalloc(&p, std::max<size_t>(bytes, 16)) != cudaSuccess) return nullptr;
        owned.push_back(p);
        return p;
    };
    const size_t n1 = size_t(MLP_H) * MLP_D0, n2 = size_t(MLP_H) * MLP_H, nb = 2 * MLP_H + MLP_H + 1;
    // f32 masters: W1, W2, then b1, b2, w3, b3; gradients and Adam moments alike
    nparams = n1 + n2 + nb;
    master = static_cast<float*>(alloc(nparams * 4));
    grad = static_cast<float*>(alloc(nparams * 4));
    m1 = static_cast<float*>(alloc(nparams * 4));
    m2 = static_cast<float*>(alloc(nparams * 4));
    w1b = static_cast<__nv_bfloat16*>(alloc(n1 * 2));
    w2b = static_cast<__nv_bfloat16*>(alloc(n2 * 2));
    w2t = static_cast<__nv_bfloat16*>(alloc(n2 * 2));
    if (!master || !grad || !m1 || !m2 || !w1b || !w2b || !w2t) return false;
    // He-uniform initialisation from a splitmix64 stream (deterministic in the seed)
    std::vector<float> h(nparams, 0.f);
    uint64_t st = seed;
    auto uni = [&]() {
        st += 0x9E3779B97F4A7C15ull;
        uint64_t z = st;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return float(double(z >> 11) * (1.0 / 9007199254740992.0)) * 2.f - 1.f;
    };
    const float s1 = std::sqrt(6.f / MLP_D0), s2 = std::sqrt(6.f / MLP_H), s3 = std::sqrt(6.f / MLP_H);
    for (size_t k = 0; k < n1; ++k) h[k] = uni() * s1;
    for (size_t k = 0; k < n2; ++k) h[n1 + k] = uni() * s2;
    for (int k = 0; k < MLP_H; ++k) h[n1 + n2 + 2 * MLP_H + k] = uni() * s3;
    return set_params(h.data()) == 0 && cudaMemset(m1, 0, nparams * 4) == cudaSuccess &&
           cudaMemset(m2, 0, nparams * 4) == cudaSuccess;
}

int Mlp::set_params(const float* host) {
    if (cudaMemcpy(master, host, nparams * 4, cudaMemcpyHostToDevice) != cudaSuccess) return -1;
    return refresh_bf16(nullptr);
}

int Mlp::refresh_bf16(cudaStream_t s) {
    const int n1 = MLP_H * MLP_D0, n2 = MLP_H * MLP_H;
    cast_bf16_kernel<<<256, 256, 0, s>>>(master, n1, w1b, nullptr, MLP_D0);
    cast_bf16_kernel<<<64, 256, 0, s>>>(master + n1, n2, w2b, w2t, MLP_H);
    return cudaStreamSynchronize(s) == cudaSuccess ? 0 : -1;
}

bool Mlp::reserve(int B) {
    if (B <= cap) return true;
    auto alloc = [&](size_t bytes) -> void* {
        void* p = nullptr;
        if (cudaMalloc(&p, std::max<size_t>(bytes, 16)) != cudaSuccess) return nullptr;
        owned.push_back(p);
        return p;
    };
    const size_t b = size_t(B);
    h1 = static_cast<__nv_bfloat16*>(alloc(b * MLP_H * 2));
    h1t = static_cast<__nv_bfloat16*>(alloc(b * MLP_H * 2));
    h2 = static_cast<__nv_bfloat16*>(alloc(b * MLP_H * 2));
    z3 = static_cast<float*>(alloc(b * 4));
    dz2 = static_cast<__nv_bfloat16*>(alloc(b * MLP_H * 2));
    dz2t = static_cast<__nv_bfloat16*>(alloc(b * MLP_H * 2));
    dz1 = static_cast<__nv_bfloat16*>(alloc(b * MLP_H * 2));
    dz1t = static_cast<__nv_bfloat16*>(alloc(b * MLP_H * 2));
    xt = static_cast<__nv_bfloat16*>(alloc(b * MLP_D0 * 2));
    lossd = static_cast<float*>(alloc(4));
    if (!h1 || !h1t || !h2 || !z3 || !dz2 || !dz2t || !dz1 || !dz1t || !xt || !lossd) return false;
    cap = B;
    return true;
}

int Mlp::forward(cudaStream_t s, const __nv_bfloat16* x, int B, float* p) {
    if (B % 64 || !reserve(B)) { set_error("forward: batch not a multiple of 64 or allocation failed"); return -1; }
    const float* b1 = master + size_t(MLP_H) * MLP_D0 + size_t(MLP_H) * MLP_H;
    const float* b2 = b1 + MLP_H;
    const float* w3 = b2 + MLP_H;
    const float* b3 = w3 + MLP_H;
    if (gemm(s, x, MLP_D0, w1b, MLP_D0, B, MLP_H, MLP_D0, EPI_BIAS | EPI_RELU, b1, nullptr, 0, nullptr, 0, h1, MLP_H, h1t, B)) return -1;
    if (gemm(s, h1, MLP_H, w2b, MLP_H, B, MLP_H, MLP_H, EPI_BIAS | EPI_RELU, b2, nullptr, 0, nullptr, 0, h2, MLP_H, nullptr, 0)) return -1;
    head_forward_kernel<<<(B + 7) / 8, 256, 0, s>>>(h2, w3, b3, B, z3, p);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int Mlp::backward(cudaStream_t s, const __nv_bfloat16* x, const float* y, const float* w, float wsum, int B, float* loss) {
    if (!reserve(B)) return -1;
    const size_t n1 = size_t(MLP_H) * MLP_D0, n2 = size_t(MLP_H) * MLP_H;
    const float* w3 = master + n1 + n2 + 2 * MLP_H;
    float* g1 = grad;
    float* g2 = grad + n1;
    float* gb1 = grad + n1 + n2;
    float* gb2 = gb1 + MLP_H;
    float* gw3 = gb2 + MLP_H;
    float* gb3 = gw3 + MLP_H;
    cudaMemsetAsync(gw3, 0, (MLP_H + 1) * 4, s);
    cudaMemsetAsync(lossd, 0, 4, s);
    head_backward_kernel<<<(B + 7) / 8, 256, 0, s>>>(h2, z3, y, w, wsum, w3, B, gw3, gb3, dz2, dz2t, lossd);
    // dW2 = dz2^T h1, db2 = colsum(dz2)
    if (gemm(s, dz2t, B, h1t, B, MLP_H, MLP_H, B, 0, nullptr, nullptr, 0, g2, MLP_H, nullptr, 0, nullptr, 0)) return -1;
    colsum_kernel<<<1, MLP_H, 0, s>>>(dz2, B, MLP_H, gb2);
    // dz1 = (dz2 W2) * (h1 > 0)
    if (gemm(s, dz2, MLP_H, w2t, MLP_H, B, MLP_H, MLP_H, EPI_MASK, nullptr, h1, MLP_H, nullptr, 0, dz1, MLP_H, dz1t, B)) return -1;
    colsum_kernel<<<1, MLP_H, 0, s>>>(dz1, B, MLP_H, gb1);
    // dW1 = dz1^T x
    transpose_bf16_kernel<<<dim3(MLP_D0 / 32, B / 32), dim3(32, 8), 0, s>>>(x, B, MLP_D0, xt);
    if (gemm(s, dz1t, B, xt, B, MLP_H, MLP_D0, B, 0, nullptr, nullptr, 0, g1, MLP_D0, nullptr, 0, nullptr, 0)) return -1;
    if (loss) cudaMemcpyAsync(loss, lossd, 4, cudaMemcpyDeviceToHost, s);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int Mlp::adam(cudaStream_t s, float lr) {
    ++step;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float c1 = 1.f - std::pow(b1, float(step)), c2 = 1.f - std::pow(b2, float(step));
    const int n1 = MLP_H * MLP_D0, n2 = MLP_H * MLP_H;
    adam_kernel<<<512, 256, 0, s>>>(master, grad, m1, m2, n1, lr, b1, b2, eps, c1, c2, w1b, nullptr, MLP_D0);
    adam_kernel<<<64, 256, 0, s>>>(master + n1, grad + n1, m1 + n1, m2 + n1, n2, lr, b1, b2, eps, c1, c2, w2b, w2t, MLP_H);
    const int nb = int(nparams) - n1 - n2;
    adam_kernel<<<1, 256, 0, s>>>(master + n1 + n2, grad + n1 + n2, m1 + n1 + n2, m2 + n1 + n2, nb, lr, b1, b2, eps, c1, c2,
                                  nullptr, nullptr, 1);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace pcbg
