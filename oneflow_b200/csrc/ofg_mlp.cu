// Coordinate MLP for warm-starting steady solves: BF16 weights and
// activations on the tensor cores (warp-level WMMA 16x16x16 BF16 tiles with
// FP32 accumulation), FP32 master weights, Adam.  Not part of the reference:
// it learns flow fields from solutions this solver produced, and the
// cold-started solve remains the fallback and the judge of convergence.
//
// Network: n_in -> width (GELU) -> ... (depth hidden layers) -> n_out.  Every
// matrix dimension is padded to a multiple of 16; padded inputs are zero and
// padded outputs carry no loss, so the padding never changes the result.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <mma.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <random>
#include <type_traits>
#include <string>
#include <vector>

#include "../../include/oneflow_b200.h"

namespace {

using bf16 = __nv_bfloat16;
constexpr int GT = 128;        // threads of a GEMM block: 4 warps
constexpr int TM = 64, TN = 64;  // block tile
constexpr int SPLITK = 32;     // batch chunks of the weight-gradient GEMMs

inline int pad16(int v) { return (v + 15) / 16 * 16; }

// C[M x N] (fp32, row-major, ldc) = op(A)[M x K] * op(B)[K x N] over the
// K range [k0, k1) of blockIdx.z's chunk.  op(A): A row-major (lda), or, with
// AT, the transpose of a row-major [K x M] array.  op(B): B row-major [K x N],
// or, with BT, the transpose of a row-major [N x K] array.  Warp w of the
// block computes rows [16 w, 16 w + 16) of the block tile, four 16x16 tiles.
template <bool AT, bool BT>
__global__ void __launch_bounds__(GT) k_gemm(int M, int N, int K, int kchunk, const bf16 *__restrict__ A, int lda,
                                             const bf16 *__restrict__ B, int ldb, float *C, int ldc,
                                             size_t zstride) {
    using namespace nvcuda;
    int warp = threadIdx.x >> 5;
    int row0 = blockIdx.y * TM + warp * 16, col0 = blockIdx.x * TN;
    if (row0 >= M) return;
    int k0 = blockIdx.z * kchunk, k1 = min(K, k0 + kchunk);
    C += blockIdx.z * zstride;
    wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) wmma::fill_fragment(acc[j], 0.0f);
    using LA = typename std::conditional<AT, wmma::col_major, wmma::row_major>::type;
    using LB = typename std::conditional<BT, wmma::col_major, wmma::row_major>::type;
    wmma::fragment<wmma::matrix_a, 16, 16, 16, bf16, LA> fa;
    wmma::fragment<wmma::matrix_b, 16, 16, 16, bf16, LB> fb;
    for (int k = k0; k < k1; k += 16) {
        const bf16 *pa = AT ? A + (size_t)k * lda + row0 : A + (size_t)row0 * lda + k;
        wmma::load_matrix_sync(fa, pa, lda);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            int c = col0 + 16 * j;
            if (c >= N) break;
            const bf16 *pb = BT ? B + (size_t)c * ldb + k : B + (size_t)k * ldb + c;
            wmma::load_matrix_sync(fb, pb, ldb);
            wmma::mma_sync(acc[j], fa, fb, acc[j]);
        }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        int c = col0 + 16 * j;
        if (c >= N) break;
        wmma::store_matrix_sync(C + (size_t)row0 * ldc + c, acc[j], ldc, wmma::mem_row_major);
    }
}

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
    return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// Z += bias; H = bf16(GELU(Z))
__global__ void k_bias_gelu(int64_t total, int N, float *Z, const float *bias, bf16 *H) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= total) return;
    float z = Z[i] + bias[i % N];
    Z[i] = z;
    H[i] = __float2bfloat16(gelu(z));
}

// output layer: Y = Z + bias; with a target, dZ = 2 (Y - T) / (rows * nout) on
// the nout real columns (0 on padding) and the row's squared error
__global__ void k_output(int rows, int N, int nout, float *Z, const float *bias, const float *T, bf16 *dZ,
                         float *rowErr) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    float e = 0.0f;
    for (int c = 0; c < N; ++c) {
        float y = Z[(size_t)r * N + c] + bias[c];
        Z[(size_t)r * N + c] = y;
        if (T) {
            float g = 0.0f;
            if (c < nout) {
                float d = y - T[(size_t)r * nout + c];
                e += d * d;
                g = 2.0f * d / float(rows * nout);
            }
            dZ[(size_t)r * N + c] = __float2bfloat16(g);
        }
    }
    if (rowErr) rowErr[r] = e;
}

// dZprev = bf16(dH * GELU'(Zprev))
__global__ void k_gelu_back(int64_t total, const float *dH, const float *Zprev, bf16 *dZ) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= total) return;
    dZ[i] = __float2bfloat16(dH[i] * gelu_grad(Zprev[i]));
}

// column sums of a bf16 [rows x N] matrix (bias gradient), one block per
// column, fixed order
__global__ void k_colsum(int rows, int N, const bf16 *dZ, float *out) {
    __shared__ float s[256];
    int c = blockIdx.x;
    float a = 0.0f;
    for (int r = threadIdx.x; r < rows; r += blockDim.x) a += __bfloat162float(dZ[(size_t)r * N + c]);
    s[threadIdx.x] = a;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[c] = s[0];
}

// sum of the split-K partials in chunk order
__global__ void k_reduce_parts(int64_t n, int parts, const float *part, float *out) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    float a = 0.0f;
    for (int p = 0; p < parts; ++p) a += part[(size_t)p * n + i];
    out[i] = a;
}

// Adam on the FP32 master copy, BF16 working copy refreshed; padded entries
// (mask 0) stay zero
__global__ void k_adam(int64_t n, float *w, float *m, float *v, const float *g, const unsigned char *mask,
                       bf16 *wb, float lr, float b1, float b2, float eps, float c1, float c2) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n || (mask && !mask[i])) return;
    float gi = g[i];
    float mi = b1 * m[i] + (1.0f - b1) * gi;
    float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi; v[i] = vi;
    float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    if (wb) wb[i] = __float2bfloat16(wi);
}

// minibatch rows: row r of step s takes sample hash(seed, s, r) mod n
__device__ __forceinline__ uint64_t mix64(uint64_t x) {
    x ^= x >> 30; x *= 0xbf58476d1ce4e5b9ULL; x ^= x >> 27; x *= 0x94d049bb133111ebULL; x ^= x >> 31;
    return x;
}
__global__ void k_gather(int rows, int64_t n, int nin, int K0, int nout, const float *X, const float *Y,
                         uint64_t seed, uint64_t step, bf16 *Xb, float *Tb) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    int64_t s = int64_t(mix64(seed ^ mix64(step * 0x9e3779b97f4a7c15ULL + uint64_t(r))) % uint64_t(n));
    for (int c = 0; c < K0; ++c) Xb[(size_t)r * K0 + c] = __float2bfloat16(c < nin ? X[s * nin + c] : 0.0f);
    for (int c = 0; c < nout; ++c) Tb[(size_t)r * nout + c] = Y[s * nout + c];
}

// rows [r0, r0 + rows) of X as a zero-padded bf16 block
__global__ void k_pack_rows(int rows, int64_t n, int64_t r0, int nin, int K0, const float *X, bf16 *Xb) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    int64_t s = r0 + r;
    for (int c = 0; c < K0; ++c)
        Xb[(size_t)r * K0 + c] = __float2bfloat16(c < nin && s < n ? X[s * nin + c] : 0.0f);
}

__global__ void k_unpack_rows(int rows, int64_t n, int64_t r0, int N, int nout, const float *Z, float *Y) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows || r0 + r >= n) return;
    for (int c = 0; c < nout; ++c) Y[(r0 + r) * nout + c] = Z[(size_t)r * N + c];
}

}  // namespace

struct ofg_mlp {
    int nin, width, depth, nout, L;
    std::vector<int> K, N;             // padded fan-in / fan-out per layer
    std::vector<int> kin, nfo;         // real fan-in / fan-out
    std::vector<size_t> woff, boff;    // offsets of each layer's W [K x N] and b [N] in the parameter arrays
    size_t nw = 0, nb = 0;
    float *w = nullptr, *b = nullptr;                // FP32 master
    bf16 *wb = nullptr;                              // BF16 working weights
    float *mw = nullptr, *vw = nullptr, *mb = nullptr, *vb = nullptr, *gw = nullptr, *gb = nullptr;
    unsigned char *wmask = nullptr, *bmask = nullptr;
    int capRows = 0;
    std::vector<float *> Z;                          // pre-activations [rows x N_l]
    std::vector<bf16 *> H;                           // inputs of each layer [rows x K_l]
    bf16 *dZ = nullptr, *dHb = nullptr;              // [rows x maxdim]
    float *dH = nullptr, *part = nullptr, *Tb = nullptr, *rowErr = nullptr;
    long long adamStep = 0;
    std::string err;
    int fail(int code, const std::string &m) { err = m; return code; }
};

namespace {

#define MCK(call)                                                                                  \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) return m->fail(OFG_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

void free_work(ofg_mlp *m) {
    for (auto p : m->Z) cudaFree(p);
    for (auto p : m->H) cudaFree(p);
    m->Z.clear(); m->H.clear();
    cudaFree(m->dZ); cudaFree(m->dHb); cudaFree(m->dH); cudaFree(m->part); cudaFree(m->Tb); cudaFree(m->rowErr);
    m->dZ = m->dHb = nullptr; m->dH = m->part = m->Tb = m->rowErr = nullptr;
    m->capRows = 0;
}

int ensure_work(ofg_mlp *m, int rows) {
    if (rows <= m->capRows) return OFG_OK;
    free_work(m);
    int maxd = 0;
    for (int l = 0; l < m->L; ++l) maxd = std::max(maxd, std::max(m->K[l], m->N[l]));
    m->Z.assign(m->L, nullptr); m->H.assign(m->L, nullptr);
    for (int l = 0; l < m->L; ++l) {
        MCK(cudaMalloc(&m->Z[l], (size_t)rows * m->N[l] * sizeof(float)));
        MCK(cudaMalloc(&m->H[l], (size_t)rows * m->K[l] * sizeof(bf16)));
    }
    MCK(cudaMalloc(&m->dZ, (size_t)rows * maxd * sizeof(bf16)));
    MCK(cudaMalloc(&m->dHb, (size_t)rows * maxd * sizeof(bf16)));
    MCK(cudaMalloc(&m->dH, (size_t)rows * maxd * sizeof(float)));
    MCK(cudaMalloc(&m->part, (size_t)SPLITK * maxd * maxd * sizeof(float)));
    MCK(cudaMalloc(&m->Tb, (size_t)rows * m->nout * sizeof(float)));
    MCK(cudaMalloc(&m->rowErr, (size_t)rows * sizeof(float)));
    m->capRows = rows;
    return OFG_OK;
}

inline unsigned blocks(int64_t n, int t) { return unsigned((n + t - 1) / t); }

// forward through every layer for `rows` rows already packed in H[0]; with a
// target Tb, the output gradient and per-row errors as well
int forward(ofg_mlp *m, int rows, bool withTarget) {
    for (int l = 0; l < m->L; ++l) {
        dim3 g(blocks(m->N[l], TN), blocks(rows, TM), 1);
        k_gemm<false, false><<<g, GT>>>(rows, m->N[l], m->K[l], m->K[l], m->H[l], m->K[l], m->wb + m->woff[l],
                                        m->N[l], m->Z[l], m->N[l], 0);
        if (l + 1 < m->L) {
            int64_t tot = (int64_t)rows * m->N[l];
            k_bias_gelu<<<blocks(tot, 256), 256>>>(tot, m->N[l], m->Z[l], m->b + m->boff[l], m->H[l + 1]);
        } else {
            k_output<<<blocks(rows, 128), 128>>>(rows, m->N[l], m->nout, m->Z[l], m->b + m->boff[l],
                                                 withTarget ? m->Tb : nullptr, m->dZ, m->rowErr);
        }
    }
    MCK(cudaGetLastError());
    return OFG_OK;
}

// gradients of the mean squared error into gw, gb (after forward with target)
int backward(ofg_mlp *m, int rows) {
    for (int l = m->L - 1; l >= 0; --l) {
        int K = m->K[l], N = m->N[l];
        // dW = H^T dZ, split over the rows, partials summed in order
        int chunk = pad16((rows + SPLITK - 1) / SPLITK);
        int parts = (rows + chunk - 1) / chunk;
        dim3 g(blocks(N, TN), blocks(K, TM), parts);
        k_gemm<true, false><<<g, GT>>>(K, N, rows, chunk, m->H[l], K, m->dZ, N, m->part, N, (size_t)K * N);
        k_reduce_parts<<<blocks((int64_t)K * N, 256), 256>>>((int64_t)K * N, parts, m->part, m->gw + m->woff[l]);
        k_colsum<<<N, 256>>>(rows, N, m->dZ, m->gb + m->boff[l]);
        if (l > 0) {
            // dH = dZ W^T, then through the GELU of the layer below
            dim3 g2(blocks(K, TN), blocks(rows, TM), 1);
            k_gemm<false, true><<<g2, GT>>>(rows, K, N, N, m->dZ, N, m->wb + m->woff[l], N, m->dH, K, 0);
            int64_t tot = (int64_t)rows * K;
            k_gelu_back<<<blocks(tot, 256), 256>>>(tot, m->dH, m->Z[l - 1], m->dZ);
        }
    }
    MCK(cudaGetLastError());
    return OFG_OK;
}

}  // namespace

extern "C" {

int ofg_mlp_create(int n_in, int width, int depth, int n_out, uint64_t seed, ofg_mlp **out) {
    if (!out || n_in < 1 || width < 16 || width % 16 || depth < 1 || n_out < 1 || n_in > 4096 || width > 4096 ||
        n_out > 4096)
        return OFG_E_ARG;
    auto *m = new ofg_mlp();
    m->nin = n_in; m->width = width; m->depth = depth; m->nout = n_out; m->L = depth + 1;
    for (int l = 0; l < m->L; ++l) {
        int fi = l == 0 ? n_in : width, fo = l + 1 < m->L ? width : n_out;
        m->kin.push_back(fi); m->nfo.push_back(fo);
        m->K.push_back(pad16(fi)); m->N.push_back(pad16(fo));
        m->woff.push_back(m->nw); m->boff.push_back(m->nb);
        m->nw += (size_t)pad16(fi) * pad16(fo); m->nb += pad16(fo);
    }
    // weights U(-1/sqrt(fan_in), 1/sqrt(fan_in)) from a seeded generator, biases 0
    std::vector<float> w(m->nw, 0.0f), b(m->nb, 0.0f);
    std::vector<unsigned char> wm(m->nw, 0), bm(m->nb, 0);
    std::mt19937_64 gen(seed);
    for (int l = 0; l < m->L; ++l) {
        float a = 1.0f / std::sqrt(float(m->kin[l]));
        std::uniform_real_distribution<float> u(-a, a);
        for (int i = 0; i < m->kin[l]; ++i)
            for (int j = 0; j < m->nfo[l]; ++j) {
                size_t k = m->woff[l] + (size_t)i * m->N[l] + j;
                w[k] = u(gen); wm[k] = 1;
            }
        for (int j = 0; j < m->nfo[l]; ++j) bm[m->boff[l] + j] = 1;
    }
    std::vector<bf16> wb(m->nw);
    for (size_t i = 0; i < m->nw; ++i) wb[i] = __float2bfloat16(w[i]);
    auto fail = [&](cudaError_t e) { ofg_mlp_destroy(m); return e == cudaErrorMemoryAllocation ? OFG_E_NOMEM : OFG_E_CUDA; };
    cudaError_t e;
    float **fp[] = {&m->w, &m->mw, &m->vw, &m->gw};
    for (float **p : fp) if ((e = cudaMalloc(p, m->nw * sizeof(float))) != cudaSuccess) return fail(e);
    float **bp[] = {&m->b, &m->mb, &m->vb, &m->gb};
    for (float **p : bp) if ((e = cudaMalloc(p, m->nb * sizeof(float))) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&m->wb, m->nw * sizeof(bf16))) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&m->wmask, m->nw)) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&m->bmask, m->nb)) != cudaSuccess) return fail(e);
    cudaMemcpy(m->w, w.data(), m->nw * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(m->wb, wb.data(), m->nw * sizeof(bf16), cudaMemcpyHostToDevice);
    cudaMemcpy(m->b, b.data(), m->nb * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(m->wmask, wm.data(), m->nw, cudaMemcpyHostToDevice);
    cudaMemcpy(m->bmask, bm.data(), m->nb, cudaMemcpyHostToDevice);
    for (float *p : {m->mw, m->vw, m->gw}) cudaMemset(p, 0, m->nw * sizeof(float));
    for (float *p : {m->mb, m->vb, m->gb}) cudaMemset(p, 0, m->nb * sizeof(float));
    if ((e = cudaDeviceSynchronize()) != cudaSuccess) return fail(e);
    *out = m;
    return OFG_OK;
}

void ofg_mlp_destroy(ofg_mlp *m) {
    if (!m) return;
    cudaDeviceSynchronize();
    free_work(m);
    for (void *p : {(void *)m->w, (void *)m->b, (void *)m->wb, (void *)m->mw, (void *)m->vw, (void *)m->mb,
                    (void *)m->vb, (void *)m->gw, (void *)m->gb, (void *)m->wmask, (void *)m->bmask})
        cudaFree(p);
    delete m;
}

const char *ofg_mlp_last_error(const ofg_mlp *m) { return m ? m->err.c_str() : "null network"; }

int64_t ofg_mlp_num_params(const ofg_mlp *m) {
    if (!m) return -1;
    int64_t n = 0;
    for (int l = 0; l < m->L; ++l) n += (int64_t)m->kin[l] * m->nfo[l] + m->nfo[l];
    return n;
}

// parameters as one FP32 host array: per layer W [fan_in][fan_out] then b [fan_out]
int ofg_mlp_get_params(ofg_mlp *m, float *out) {
    if (!m || !out) return OFG_E_ARG;
    std::vector<float> w(m->nw), b(m->nb);
    MCK(cudaMemcpy(w.data(), m->w, m->nw * sizeof(float), cudaMemcpyDeviceToHost));
    MCK(cudaMemcpy(b.data(), m->b, m->nb * sizeof(float), cudaMemcpyDeviceToHost));
    size_t o = 0;
    for (int l = 0; l < m->L; ++l) {
        for (int i = 0; i < m->kin[l]; ++i)
            for (int j = 0; j < m->nfo[l]; ++j) out[o++] = w[m->woff[l] + (size_t)i * m->N[l] + j];
        for (int j = 0; j < m->nfo[l]; ++j) out[o++] = b[m->boff[l] + j];
    }
    return OFG_OK;
}

int ofg_mlp_set_params(ofg_mlp *m, const float *in) {
    if (!m || !in) return OFG_E_ARG;
    std::vector<float> w(m->nw, 0.0f), b(m->nb, 0.0f);
    size_t o = 0;
    for (int l = 0; l < m->L; ++l) {
        for (int i = 0; i < m->kin[l]; ++i)
            for (int j = 0; j < m->nfo[l]; ++j) w[m->woff[l] + (size_t)i * m->N[l] + j] = in[o++];
        for (int j = 0; j < m->nfo[l]; ++j) b[m->boff[l] + j] = in[o++];
    }
    std::vector<bf16> wb(m->nw);
    for (size_t i = 0; i < m->nw; ++i) wb[i] = __float2bfloat16(w[i]);
    MCK(cudaMemcpy(m->w, w.data(), m->nw * sizeof(float), cudaMemcpyHostToDevice));
    MCK(cudaMemcpy(m->wb, wb.data(), m->nw * sizeof(bf16), cudaMemcpyHostToDevice));
    MCK(cudaMemcpy(m->b, b.data(), m->nb * sizeof(float), cudaMemcpyHostToDevice));
    for (float *p : {m->mw, m->vw}) MCK(cudaMemset(p, 0, m->nw * sizeof(float)));
    for (float *p : {m->mb, m->vb}) MCK(cudaMemset(p, 0, m->nb * sizeof(float)));
    m->adamStep = 0;
    return OFG_OK;
}

// Y[n][n_out] = f(X[n][n_in]) (device arrays, FP32), in blocks of `rows`
int ofg_mlp_predict(ofg_mlp *m, const float *x, int64_t n, float *y) {
    if (!m || !x || !y || n < 0) return OFG_E_ARG;
    const int rows = 16384;
    int rc = ensure_work(m, rows);
    if (rc) return rc;
    for (int64_t r0 = 0; r0 < n; r0 += rows) {
        int rr = int(std::min<int64_t>(rows, n - r0));
        int rp = (rr + TM - 1) / TM * TM;
        k_pack_rows<<<blocks(rp, 128), 128>>>(rp, n, r0, m->nin, m->K[0], x, m->H[0]);
        if ((rc = forward(m, rp, false))) return rc;
        k_unpack_rows<<<blocks(rp, 128), 128>>>(rp, n, r0, m->N[m->L - 1], m->nout, m->Z[m->L - 1], y);
    }
    MCK(cudaGetLastError());
    MCK(cudaDeviceSynchronize());
    return OFG_OK;
}

// Mean squared error of the batch X[n], Y[n] (n a multiple of 64, at most
// 65,536) and its gradient (host arrays in the parameter layout); no update
int ofg_mlp_loss_grad(ofg_mlp *m, const float *x, const float *y, int64_t n, float *loss, float *grad) {
    if (!m || !x || !y || n <= 0 || n % TM || n > 65536) return OFG_E_ARG;
    int rows = int(n);
    int rc = ensure_work(m, rows);
    if (rc) return rc;
    k_pack_rows<<<blocks(rows, 128), 128>>>(rows, n, 0, m->nin, m->K[0], x, m->H[0]);
    MCK(cudaMemcpy(m->Tb, y, (size_t)rows * m->nout * sizeof(float), cudaMemcpyDeviceToDevice));
    if ((rc = forward(m, rows, true)) || (rc = backward(m, rows))) return rc;
    std::vector<float> e(rows), gw(m->nw), gb(m->nb);
    MCK(cudaMemcpy(e.data(), m->rowErr, rows * sizeof(float), cudaMemcpyDeviceToHost));
    MCK(cudaMemcpy(gw.data(), m->gw, m->nw * sizeof(float), cudaMemcpyDeviceToHost));
    MCK(cudaMemcpy(gb.data(), m->gb, m->nb * sizeof(float), cudaMemcpyDeviceToHost));
    double s = 0.0;
    for (float v : e) s += v;
    if (loss) *loss = float(s / (double(rows) * m->nout));
    if (grad) {
        size_t o = 0;
        for (int l = 0; l < m->L; ++l) {
            for (int i = 0; i < m->kin[l]; ++i)
                for (int j = 0; j < m->nfo[l]; ++j) grad[o++] = gw[m->woff[l] + (size_t)i * m->N[l] + j];
            for (int j = 0; j < m->nfo[l]; ++j) grad[o++] = gb[m->boff[l] + j];
        }
    }
    return OFG_OK;
}

// `steps` Adam steps on minibatches of `batch` rows (a multiple of 64) drawn
// from X[n], Y[n] (device, FP32); loss_out (host, may be NULL) receives each
// step's minibatch loss
int ofg_mlp_train(ofg_mlp *m, const float *x, const float *y, int64_t n, int batch, int steps, float lr,
                  uint64_t seed, float *loss_out) {
    if (!m || !x || !y || n <= 0 || batch <= 0 || batch % TM || batch > 65536 || steps < 0) return OFG_E_ARG;
    int rc = ensure_work(m, batch);
    if (rc) return rc;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    std::vector<float> e(batch);
    for (int s = 0; s < steps; ++s) {
        k_gather<<<blocks(batch, 128), 128>>>(batch, n, m->nin, m->K[0], m->nout, x, y, seed, uint64_t(s), m->H[0],
                                              m->Tb);
        if ((rc = forward(m, batch, true)) || (rc = backward(m, batch))) return rc;
        ++m->adamStep;
        float c1 = 1.0f - std::pow(b1, float(m->adamStep)), c2 = 1.0f - std::pow(b2, float(m->adamStep));
        k_adam<<<blocks(m->nw, 256), 256>>>(m->nw, m->w, m->mw, m->vw, m->gw, m->wmask, m->wb, lr, b1, b2, eps, c1, c2);
        k_adam<<<blocks(m->nb, 256), 256>>>(m->nb, m->b, m->mb, m->vb, m->gb, m->bmask, nullptr, lr, b1, b2, eps, c1,
                                            c2);
        if (loss_out) {
            MCK(cudaMemcpy(e.data(), m->rowErr, batch * sizeof(float), cudaMemcpyDeviceToHost));
            double t = 0.0;
            for (float v : e) t += v;
            loss_out[s] = float(t / (double(batch) * m->nout));
        }
    }
    MCK(cudaGetLastError());
    MCK(cudaDeviceSynchronize());
    return OFG_OK;
}

}  // extern "C"
