// A small multilayer perceptron trained and evaluated with hand-written
// kernels: the learned initial guess of the strong fluid-structure coupling
// iteration (no counterpart in the reference, whose coupling is explicit).
//
//   x (n_in) -> tanh(W1 x + b1) (64) -> tanh(W2 h1 + b2) (64) -> W3 h2 + b3 (n_out)
//
// FP32 throughout.  Parameters are one flat array [W1 b1 W2 b2 W3 b3] with
// W[out][in] row-major.  Loss: mean over the samples of the summed squared
// output errors.  Gradients are accumulated per block in a fixed order and
// summed over blocks in a fixed order, so training is deterministic.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <new>
#include <random>
#include <vector>

#include "../../include/fribois2d.h"

namespace {

constexpr int kH = 64;      // hidden width
constexpr int kMaxIn = 64;  // input width limit
constexpr int kMaxOut = 8;  // output width limit
constexpr int kS = 16;      // samples per block

struct Shape {
    int nin, nout;
    int oW1, ob1, oW2, ob2, oW3, ob3, n;
    explicit Shape(int ni = 0, int no = 0) : nin(ni), nout(no) {
        oW1 = 0;
        ob1 = oW1 + kH * nin;
        oW2 = ob1 + kH;
        ob2 = oW2 + kH * kH;
        oW3 = ob2 + kH;
        ob3 = oW3 + nout * kH;
        n = ob3 + nout;
    }
};

// forward pass of kS samples per block (64 threads: one per hidden unit);
// H1, H2 keep the activations for the backward pass (may be null)
__global__ void __launch_bounds__(kH) k_mlp_fwd(Shape sh, const float *__restrict__ P, const float *__restrict__ X,
                                                 int B, float *__restrict__ H1, float *__restrict__ H2,
                                                 float *__restrict__ Y) {
    __shared__ float xs[kS][kMaxIn];
    __shared__ float h1[kS][kH], h2[kS][kH];
    const int t = threadIdx.x, s0 = blockIdx.x * kS;
    const int ns = min(kS, B - s0);
    for (int i = t; i < kS * sh.nin; i += kH) {
        const int s = i / sh.nin, k = i - s * sh.nin;
        xs[s][k] = (s < ns) ? X[static_cast<size_t>(s0 + s) * sh.nin + k] : 0.0f;
    }
    __syncthreads();
    const float *w1 = P + sh.oW1 + t * sh.nin;
    for (int s = 0; s < kS; ++s) {
        float a = P[sh.ob1 + t];
        for (int k = 0; k < sh.nin; ++k) a = fmaf(w1[k], xs[s][k], a);
        h1[s][t] = tanhf(a);
    }
    __syncthreads();
    const float *w2 = P + sh.oW2 + t * kH;
    for (int s = 0; s < kS; ++s) {
        float a = P[sh.ob2 + t];
        for (int k = 0; k < kH; ++k) a = fmaf(w2[k], h1[s][k], a);
        h2[s][t] = tanhf(a);
    }
    __syncthreads();
    for (int i = t; i < ns * kH; i += kH) {
        const int s = i / kH, k = i - s * kH;
        if (H1) H1[static_cast<size_t>(s0 + s) * kH + k] = h1[s][k];
        if (H2) H2[static_cast<size_t>(s0 + s) * kH + k] = h2[s][k];
    }
    for (int i = t; i < ns * sh.nout; i += kH) {
        const int s = i / sh.nout, o = i - s * sh.nout;
        const float *w3 = P + sh.oW3 + o * kH;
        float a = P[sh.ob3 + o];
        for (int k = 0; k < kH; ++k) a = fmaf(w3[k], h2[s][k], a);
        Y[static_cast<size_t>(s0 + s) * sh.nout + o] = a;
    }
}

// backward pass: per-block parameter gradients (G[block][param]) and loss
// partials for the samples of the block; dL/dy = 2 (y - target) / B
__global__ void __launch_bounds__(kH) k_mlp_bwd(Shape sh, const float *__restrict__ P, const float *__restrict__ X,
                                                 const float *__restrict__ H1, const float *__restrict__ H2,
                                                 const float *__restrict__ Y, const float *__restrict__ T, int B,
                                                 float *__restrict__ G, float *__restrict__ L) {
    __shared__ float xs[kS][kMaxIn];
    __shared__ float h1[kS][kH], h2[kS][kH], d1[kS][kH], d2[kS][kH];
    __shared__ float dy[kS][kMaxOut];
    __shared__ float lsum[kH];
    const int t = threadIdx.x, s0 = blockIdx.x * kS;
    const int ns = min(kS, B - s0);
    float *g = G + static_cast<size_t>(blockIdx.x) * sh.n;
    for (int i = t; i < kS * sh.nin; i += kH) {
        const int s = i / sh.nin, k = i - s * sh.nin;
        xs[s][k] = (s < ns) ? X[static_cast<size_t>(s0 + s) * sh.nin + k] : 0.0f;
    }
    for (int i = t; i < kS * kH; i += kH) {
        const int s = i / kH, k = i - s * kH;
        h1[s][k] = (s < ns) ? H1[static_cast<size_t>(s0 + s) * kH + k] : 0.0f;
        h2[s][k] = (s < ns) ? H2[static_cast<size_t>(s0 + s) * kH + k] : 0.0f;
    }
    float l = 0.0f;
    for (int i = t; i < kS * sh.nout; i += kH) {
        const int s = i / sh.nout, o = i - s * sh.nout;
        float e = 0.0f;
        if (s < ns) e = Y[static_cast<size_t>(s0 + s) * sh.nout + o] - T[static_cast<size_t>(s0 + s) * sh.nout + o];
        dy[s][o] = 2.0f * e / static_cast<float>(B);
        l = fmaf(e, e, l);
    }
    lsum[t] = l;
    __syncthreads();
    // layer 3: dW3[o][k] = sum_s dy[s][o] h2[s][k]; db3[o] = sum_s dy[s][o]
    for (int i = t; i < sh.nout * kH; i += kH) {
        const int o = i / kH, k = i - o * kH;
        float a = 0.0f;
        for (int s = 0; s < kS; ++s) a = fmaf(dy[s][o], h2[s][k], a);
        g[sh.oW3 + i] = a;
    }
    if (t < sh.nout) {
        float a = 0.0f;
        for (int s = 0; s < kS; ++s) a += dy[s][t];
        g[sh.ob3 + t] = a;
    }
    // d2 = (W3^T dy) * (1 - h2^2)
    for (int s = 0; s < kS; ++s) {
        float a = 0.0f;
        for (int o = 0; o < sh.nout; ++o) a = fmaf(P[sh.oW3 + o * kH + t], dy[s][o], a);
        d2[s][t] = a * (1.0f - h2[s][t] * h2[s][t]);
    }
    __syncthreads();
    // layer 2: dW2[t][k] = sum_s d2[s][t] h1[s][k]
    for (int k = 0; k < kH; ++k) {
        float a = 0.0f;
        for (int s = 0; s < kS; ++s) a = fmaf(d2[s][t], h1[s][k], a);
        g[sh.oW2 + t * kH + k] = a;
    }
    {
        float a = 0.0f;
        for (int s = 0; s < kS; ++s) a += d2[s][t];
        g[sh.ob2 + t] = a;
    }
    // d1 = (W2^T d2) * (1 - h1^2)
    for (int s = 0; s < kS; ++s) {
        float a = 0.0f;
        for (int j = 0; j < kH; ++j) a = fmaf(P[sh.oW2 + j * kH + t], d2[s][j], a);
        d1[s][t] = a * (1.0f - h1[s][t] * h1[s][t]);
    }
    __syncthreads();
    for (int k = 0; k < sh.nin; ++k) {
        float a = 0.0f;
        for (int s = 0; s < kS; ++s) a = fmaf(d1[s][t], xs[s][k], a);
        g[sh.oW1 + t * sh.nin + k] = a;
    }
    {
        float a = 0.0f;
        for (int s = 0; s < kS; ++s) a += d1[s][t];
        g[sh.ob1 + t] = a;
    }
    if (t == 0) {
        float a = 0.0f;
        for (int i = 0; i < kH; ++i) a += lsum[i];
        L[blockIdx.x] = a;
    }
}

// sums the per-block partials in block order (deterministic)
__global__ void k_mlp_reduce(int n, int nb, const float *__restrict__ G, float *__restrict__ out,
                             const float *__restrict__ L, float *__restrict__ loss, int B) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        float a = 0.0f;
        for (int b = 0; b < nb; ++b) a += G[static_cast<size_t>(b) * n + i];
        out[i] = a;
    }
    if (i == 0) {
        float a = 0.0f;
        for (int b = 0; b < nb; ++b) a += L[b];
        *loss = a / static_cast<float>(B);
    }
}

// Adam (Kingma and Ba 2015) with bias correction
__global__ void k_adam(int n, float *__restrict__ P, const float *__restrict__ G, float *__restrict__ M,
                       float *__restrict__ V, float lr, float b1, float b2, float eps, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float g = G[i];
    const float m = b1 * M[i] + (1.0f - b1) * g;
    const float v = b2 * V[i] + (1.0f - b2) * g * g;
    M[i] = m;
    V[i] = v;
    P[i] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
}

}  // namespace

struct fb_mlp {
    int device = 0;
    Shape sh;
    float *P = nullptr, *M = nullptr, *V = nullptr, *G = nullptr;
    int step = 0;
    // scratch sized for cap samples
    int cap = 0;
    float *X = nullptr, *T = nullptr, *Y = nullptr, *H1 = nullptr, *H2 = nullptr, *Gb = nullptr, *Lb = nullptr,
          *loss = nullptr;
};

namespace {

#define MK(call)                                     \
    do {                                             \
        if ((call) != cudaSuccess) return FB_ERR_CUDA; \
    } while (0)

int ensure(fb_mlp *m, int B) {
    if (B <= m->cap) return FB_OK;
    cudaFree(m->X);
    cudaFree(m->T);
    cudaFree(m->Y);
    cudaFree(m->H1);
    cudaFree(m->H2);
    cudaFree(m->Gb);
    cudaFree(m->Lb);
    const int nb = (B + kS - 1) / kS;
    MK(cudaMalloc(&m->X, sizeof(float) * B * m->sh.nin));
    MK(cudaMalloc(&m->T, sizeof(float) * B * m->sh.nout));
    MK(cudaMalloc(&m->Y, sizeof(float) * B * m->sh.nout));
    MK(cudaMalloc(&m->H1, sizeof(float) * B * kH));
    MK(cudaMalloc(&m->H2, sizeof(float) * B * kH));
    MK(cudaMalloc(&m->Gb, sizeof(float) * static_cast<size_t>(nb) * m->sh.n));
    MK(cudaMalloc(&m->Lb, sizeof(float) * nb));
    m->cap = B;
    return FB_OK;
}

// forward + backward + block reduction on the B samples already in m->X, m->T
void grad_on_device(fb_mlp *m, int B) {
    const int nb = (B + kS - 1) / kS;
    k_mlp_fwd<<<nb, kH>>>(m->sh, m->P, m->X, B, m->H1, m->H2, m->Y);
    k_mlp_bwd<<<nb, kH>>>(m->sh, m->P, m->X, m->H1, m->H2, m->Y, m->T, B, m->Gb, m->Lb);
    k_mlp_reduce<<<(m->sh.n + 255) / 256, 256>>>(m->sh.n, nb, m->Gb, m->G, m->Lb, m->loss, B);
}

}  // namespace

extern "C" {

int fb_mlp_destroy(fb_mlp *m) {
    if (!m) return FB_OK;
    cudaSetDevice(m->device);
    for (float *p : {m->P, m->M, m->V, m->G, m->X, m->T, m->Y, m->H1, m->H2, m->Gb, m->Lb, m->loss}) cudaFree(p);
    delete m;
    return FB_OK;
}

int fb_mlp_create(int device, int n_in, int n_out, uint64_t seed, fb_mlp **out) {
    if (!out || n_in < 1 || n_in > kMaxIn || n_out < 1 || n_out > kMaxOut) return FB_ERR_STATE;
    *out = nullptr;
    fb_mlp *m = new (std::nothrow) fb_mlp;
    if (!m) return FB_ERR_CUDA;
    m->device = device;
    m->sh = Shape(n_in, n_out);
    if (cudaSetDevice(device) != cudaSuccess) {
        delete m;
        return FB_ERR_CUDA;
    }
    const size_t bytes = sizeof(float) * m->sh.n;
    if (cudaMalloc(&m->P, bytes) != cudaSuccess || cudaMalloc(&m->M, bytes) != cudaSuccess ||
        cudaMalloc(&m->V, bytes) != cudaSuccess || cudaMalloc(&m->G, bytes) != cudaSuccess ||
        cudaMalloc(&m->loss, sizeof(float)) != cudaSuccess) {
        fb_mlp_destroy(m);
        return FB_ERR_CUDA;
    }
    // Glorot-uniform weights, zero biases, from a seeded generator
    std::vector<float> p(static_cast<size_t>(m->sh.n), 0.0f);
    std::mt19937_64 rng(seed);
    auto fill = [&](int off, int fan_out, int fan_in) {
        const float a = std::sqrt(6.0f / static_cast<float>(fan_in + fan_out));
        std::uniform_real_distribution<float> u(-a, a);
        for (int i = 0; i < fan_out * fan_in; ++i) p[static_cast<size_t>(off + i)] = u(rng);
    };
    fill(m->sh.oW1, kH, n_in);
    fill(m->sh.oW2, kH, kH);
    fill(m->sh.oW3, n_out, kH);
    if (cudaMemcpy(m->P, p.data(), bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(m->M, 0, bytes) != cudaSuccess || cudaMemset(m->V, 0, bytes) != cudaSuccess) {
        fb_mlp_destroy(m);
        return FB_ERR_CUDA;
    }
    *out = m;
    return FB_OK;
}

int fb_mlp_params(fb_mlp *m, int *n) {
    if (!m || !n) return FB_ERR_STATE;
    *n = m->sh.n;
    return FB_OK;
}

int fb_mlp_get(fb_mlp *m, float *params) {
    if (!m || !params) return FB_ERR_STATE;
    MK(cudaSetDevice(m->device));
    MK(cudaMemcpy(params, m->P, sizeof(float) * m->sh.n, cudaMemcpyDeviceToHost));
    return FB_OK;
}

int fb_mlp_set(fb_mlp *m, const float *params) {
    if (!m || !params) return FB_ERR_STATE;
    MK(cudaSetDevice(m->device));
    MK(cudaMemcpy(m->P, params, sizeof(float) * m->sh.n, cudaMemcpyHostToDevice));
    MK(cudaMemset(m->M, 0, sizeof(float) * m->sh.n));
    MK(cudaMemset(m->V, 0, sizeof(float) * m->sh.n));
    m->step = 0;
    return FB_OK;
}

// outputs for n samples (host arrays: x n x n_in, y n x n_out)
int fb_mlp_predict(fb_mlp *m, const float *x, int n, float *y) {
    if (!m || !x || !y || n < 1) return FB_ERR_STATE;
    MK(cudaSetDevice(m->device));
    int st = ensure(m, n);
    if (st) return st;
    MK(cudaMemcpy(m->X, x, sizeof(float) * n * m->sh.nin, cudaMemcpyHostToDevice));
    k_mlp_fwd<<<(n + kS - 1) / kS, kH>>>(m->sh, m->P, m->X, n, nullptr, nullptr, m->Y);
    MK(cudaGetLastError());
    MK(cudaMemcpy(y, m->Y, sizeof(float) * n * m->sh.nout, cudaMemcpyDeviceToHost));
    return FB_OK;
}

// full-batch loss and gradient (host arrays), for checking the kernels
int fb_mlp_grad(fb_mlp *m, const float *x, const float *t, int n, float *grad, float *loss) {
    if (!m || !x || !t || n < 1 || !grad || !loss) return FB_ERR_STATE;
    MK(cudaSetDevice(m->device));
    int st = ensure(m, n);
    if (st) return st;
    MK(cudaMemcpy(m->X, x, sizeof(float) * n * m->sh.nin, cudaMemcpyHostToDevice));
    MK(cudaMemcpy(m->T, t, sizeof(float) * n * m->sh.nout, cudaMemcpyHostToDevice));
    grad_on_device(m, n);
    MK(cudaGetLastError());
    MK(cudaMemcpy(grad, m->G, sizeof(float) * m->sh.n, cudaMemcpyDeviceToHost));
    MK(cudaMemcpy(loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost));
    return FB_OK;
}

// Adam on minibatches of `batch` samples for `epochs` passes over the n
// samples (host arrays, shuffled each epoch by a seeded generator);
// loss_out (may be null) receives the mean minibatch loss of the last epoch.
int fb_mlp_train(fb_mlp *m, const float *x, const float *t, int n, int epochs, int batch, float lr, uint64_t seed,
                 float *loss_out) {
    if (!m || !x || !t || n < 1 || epochs < 1 || batch < 1) return FB_ERR_STATE;
    MK(cudaSetDevice(m->device));
    batch = std::min(batch, n);
    int st = ensure(m, batch);
    if (st) return st;
    const int ni = m->sh.nin, no = m->sh.nout;
    std::vector<int> idx(static_cast<size_t>(n));
    for (int i = 0; i < n; ++i) idx[static_cast<size_t>(i)] = i;
    std::mt19937_64 rng(seed);
    std::vector<float> bx(static_cast<size_t>(batch) * ni), bt(static_cast<size_t>(batch) * no);
    double last = 0.0;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int e = 0; e < epochs; ++e) {
        std::shuffle(idx.begin(), idx.end(), rng);
        double esum = 0.0;
        int nbt = 0;
        for (int s0 = 0; s0 + batch <= n; s0 += batch) {
            for (int r = 0; r < batch; ++r) {
                const int i = idx[static_cast<size_t>(s0 + r)];
                std::memcpy(&bx[static_cast<size_t>(r) * ni], x + static_cast<size_t>(i) * ni, sizeof(float) * ni);
                std::memcpy(&bt[static_cast<size_t>(r) * no], t + static_cast<size_t>(i) * no, sizeof(float) * no);
            }
            MK(cudaMemcpy(m->X, bx.data(), sizeof(float) * bx.size(), cudaMemcpyHostToDevice));
            MK(cudaMemcpy(m->T, bt.data(), sizeof(float) * bt.size(), cudaMemcpyHostToDevice));
            grad_on_device(m, batch);
            ++m->step;
            const float c1 = 1.0f - std::pow(b1, static_cast<float>(m->step));
            const float c2 = 1.0f - std::pow(b2, static_cast<float>(m->step));
            k_adam<<<(m->sh.n + 255) / 256, 256>>>(m->sh.n, m->P, m->G, m->M, m->V, lr, b1, b2, eps, c1, c2);
            float l = 0.0f;
            MK(cudaMemcpy(&l, m->loss, sizeof(float), cudaMemcpyDeviceToHost));
            esum += l;
            ++nbt;
        }
        last = nbt ? esum / nbt : 0.0;
    }
    MK(cudaGetLastError());
    if (loss_out) *loss_out = static_cast<float>(last);
    return FB_OK;
}

}  // extern "C"

namespace fb {
// the parameters as the coupling's device-side inference reads them
const float *mlp_params_device(const fb_mlp *m, int *n_in, int *n_out) {
    if (!m) return nullptr;
    if (n_in) *n_in = m->sh.nin;
    if (n_out) *n_out = m->sh.nout;
    return m->P;
}
}  // namespace fb
