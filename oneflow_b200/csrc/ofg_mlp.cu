// Coordinate MLP for warm-starting steady solves: BF16 weights and
// activations on the tensor cores (tcgen05.mma with FP32 accumulation in
// tensor memory), FP32 master weights, Adam.  Not part of the reference:
// it learns flow fields from solutions this solver produced, and the
// cold-started solve remains the fallback and the arbiter of convergence.
//
// Network: n_in -> width (GELU) -> ... (depth hidden layers) -> n_out.  Every
// matrix dimension is padded to a multiple of 16; padded inputs are zero and
// padded outputs carry no loss, so the padding never changes the result.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

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
constexpr int ROWS = 64;       // row granularity of the batches the API takes
constexpr int SPLITK = 32;     // batch chunks of the weight-gradient GEMMs

inline int pad16(int v) { return (v + 15) / 16 * 16; }

// ---------------------------------------------------------------------------
// GEMM on the fifth-generation tensor cores.  A CTA of four warps computes a
// BM x BN tile of C = op(A) op(B): the BF16 operand tiles of one K block
// (BM x BK of A, up to BN x BK of B) are staged in shared memory in core
// matrices without swizzle (128 bytes each, 128 B apart along K, 1,024 B apart
// along M / N; K-major or MN-major as the operand lies in memory), one
// thread issues tcgen05.mma (M 128, N the tile's width, K 16, FP32
// accumulation in tensor memory) and tcgen05.commit arrives on the stage's
// mbarrier.  The operand tiles arrive by cp.async 16-byte copies into a ring
// of four stages: the copies of the next three K blocks are in flight while
// the MMAs of the current one run.  The epilogue
// reads the accumulator with tcgen05.ld: warp w holds rows 32w..32w+31 (its
// tensor-memory lanes), 16 columns per load.  Every wait is bounded; a wait
// that runs out sets g_gemm_status and the CTA frees its tensor memory and
// returns.
// ---------------------------------------------------------------------------
constexpr int GT = 128;                       // threads of a GEMM block
constexpr int BM = 128, BN = 128, BK = 64;    // block tile
constexpr int SBO = (BK / 8) * 128;           // bytes between 8-row core-matrix groups
constexpr int NSTAGE = 4;                     // K blocks in flight
constexpr int TILE_A = BM * BK * 2, TILE_B = BN * BK * 2, STAGE = TILE_A + TILE_B;
constexpr int SMEM_GEMM = NSTAGE * STAGE + 1024 + 8 * NSTAGE + 16;   // stages, alignment slack, barriers, slot
constexpr unsigned WAIT_LIMIT = 1u << 20;     // try_wait rounds before a wait gives up

__device__ unsigned g_gemm_status;            // nonzero: a GEMM wait ran out

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// shared-memory matrix descriptor: start address, leading (K) byte offset
// 128, stride (M/N) byte offset SBO, descriptor version 1, no swizzle (the
// same fields describe the K-major and the MN-major staging)
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    return uint64_t((addr >> 4) & 0x3FFF) | (uint64_t(128 >> 4) << 16) | (uint64_t(SBO >> 4) << 32) |
           (uint64_t(1) << 46);
}

// instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, each
// K-major (0) or MN-major (1), N = n, M = BM
__device__ __forceinline__ uint32_t instr_desc(int n, uint32_t a_mn, uint32_t b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (a_mn << 15) | (b_mn << 16) | (uint32_t(n >> 3) << 17) |
           (uint32_t(BM >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint32_t bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (unsigned i = 0; i < WAIT_LIMIT; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void mma_bf16(uint32_t tmem, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t addr, uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(addr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Start the copies of rows [r0, r0 + nr) x K block [kb, kb + BK) of an
// operand whose element (r, k) is g[r * ld + k] (T false: K contiguous,
// staged K-major: a core matrix holds 8 rows x 8 K) or g[k * ld + r] (T true:
// rows contiguous, staged MN-major: a core matrix holds 8 K x 8 rows); either
// way core matrices lie 128 B apart along K and SBO apart along the rows, and
// every 16-byte chunk of the source is one 16-byte cp.async.  A warp's 32
// copies cover 512 contiguous bytes of shared memory.  Chunks of rows at or
// beyond `rows` or of K at or beyond k1 are filled with zeros (source size
// 0).  rows, nr, ld, kb and k1 are multiples of 8; nr <= 128.
template <bool T>
__device__ __forceinline__ void stage_tile(unsigned char *s, const bf16 *__restrict__ g, int ld, int rows, int r0,
                                           int nr, int kb, int k1) {
    static_assert(BK == 64, "eight 8-element K chunks per block");
    const int items = nr * (BK / 8), nc = nr >> 3;
#pragma unroll
    for (int u = 0; u < 8; ++u) {
        const int i = threadIdx.x + u * GT;
        if (i < items) {
            int r, k;   // first row and K of the chunk
            uint32_t off;
            if (!T) {   // i: row % 8, then K chunk, then row / 8
                r = (i & 7) + ((i >> 6) << 3);
                k = ((i >> 3) & 7) * 8;
                off = (r >> 3) * SBO + (k >> 3) * 128 + (r & 7) * 16;
            } else {    // i: K % 8, then row chunk, then K / 8
                k = (i & 7) + ((i >> 3) / nc) * 8;
                r = ((i >> 3) % nc) * 8;
                off = (r >> 3) * SBO + (k >> 3) * 128 + (k & 7) * 16;
            }
            const bool in = r0 + r < rows && kb + k < k1;
            const bf16 *src = in ? (T ? g + (size_t)(kb + k) * ld + r0 + r : g + (size_t)(r0 + r) * ld + kb + k) : g;
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(s + off)), "l"(src),
                         "r"(in ? 16 : 0)
                         : "memory");
        }
    }
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// C[M x N] (FP32, row-major, ldc) = op(A)[M x K] op(B)[K x N] over the K range
// [k0, k1) of blockIdx.z's chunk, into C + blockIdx.z * zstride.  op(A): A
// row-major (lda), or, with AT, the transpose of a row-major [K x M] array.
// op(B): B row-major [K x N], or, with BT, the transpose of a row-major
// [N x K] array.  M, N, K, kchunk and the leading dimensions are multiples of
// 16; the arrays are 16-byte aligned.
template <bool AT, bool BT>
__global__ void __launch_bounds__(GT, 1) k_gemm(int M, int N, int K, int kchunk, const bf16 *__restrict__ A, int lda,
                                                const bf16 *__restrict__ B, int ldb, float *C, int ldc,
                                                size_t zstride) {
    extern __shared__ unsigned char smem_raw[];
    unsigned char *sm = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                                          ~uintptr_t(1023));
    const uint32_t bar0 = smem_u32(sm + NSTAGE * STAGE), slot = smem_u32(sm + NSTAGE * STAGE + 8 * NSTAGE);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN, nt = min(BN, N - n0);
    const int k0 = blockIdx.z * kchunk, k1 = min(K, k0 + kchunk);
    const int nkb = k1 > k0 ? (k1 - k0 + BK - 1) / BK : 0;
    C += blockIdx.z * zstride;
    if (threadIdx.x == 0) {
        for (int q = 0; q < NSTAGE; ++q) mbar_init(bar0 + 8 * q);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot), "r"(BN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *reinterpret_cast<volatile uint32_t *>(sm + NSTAGE * STAGE + 8 * NSTAGE);
    const uint32_t idesc = instr_desc(nt, AT ? 1u : 0u, BT ? 0u : 1u);
    // start the copies of K block kb into its stage; one commit group per call
    // (empty past the last block), so that the group count stays uniform
    auto issue = [&](int kb) {
        if (kb < nkb) {
            unsigned char *sa = sm + (kb % NSTAGE) * STAGE;
            const int kbase = k0 + kb * BK;
            stage_tile<AT>(sa, A, lda, M, m0, BM, kbase, k1);
            stage_tile<!BT>(sa + TILE_A, B, ldb, N, n0, nt, kbase, k1);
        }
        cp_async_commit();
    };
    for (int q = 0; q < NSTAGE - 1; ++q) issue(q);
    int ok = 1, issued = 0;   // K blocks whose MMAs have been committed (the same in every thread)
    for (int kb = 0; kb < nkb; ++kb) {
        const int st = kb % NSTAGE;
        cp_async_wait<NSTAGE - 2>();                                    // this thread's copies of block kb
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // visible to the tensor core
        __syncthreads();                                                // everyone's
        if (threadIdx.x == 0) {
            tc_fence_after();
            const int nk16 = min(BK, k1 - (k0 + kb * BK)) / 16;
            const uint32_t a0 = smem_u32(sm + st * STAGE), b0 = a0 + TILE_A;
            for (int j = 0; j < nk16; ++j)
                mma_bf16(tmem, smem_desc(a0 + j * 256), smem_desc(b0 + j * 256), idesc, (kb | j) != 0);
            mma_commit(bar0 + 8 * st);
        }
        issued = kb + 1;
        // the next copies go to the stage of block kb - 1: its MMAs must be done
        if (kb >= 1) ok = mbar_wait(bar0 + 8 * ((kb - 1) % NSTAGE), ((kb - 1) / NSTAGE) & 1);
        if (!__syncthreads_and(ok)) break;
        issue(kb + NSTAGE - 1);
    }
    cp_async_wait<0>();
    // the last commit covers every MMA issued before it
    if (ok && issued > 0) ok = mbar_wait(bar0 + 8 * ((issued - 1) % NSTAGE), ((issued - 1) / NSTAGE) & 1);
    ok = __syncthreads_and(ok);
    tc_fence_after();
    if (ok) {
        const int r = m0 + warp * 32 + lane;
        for (int c = 0; c < nt; c += 16) {
            uint32_t v[16];
            if (nkb > 0) {
                tmem_ld16(tmem + (uint32_t(warp * 32) << 16) + uint32_t(c), v);
            } else {
#pragma unroll
                for (int j = 0; j < 16; ++j) v[j] = 0u;
            }
            if (r < M) {
                float4 *o = reinterpret_cast<float4 *>(C + (size_t)r * ldc + n0 + c);
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    o[j] = make_float4(__uint_as_float(v[4 * j]), __uint_as_float(v[4 * j + 1]),
                                       __uint_as_float(v[4 * j + 2]), __uint_as_float(v[4 * j + 3]));
            }
        }
    } else if (threadIdx.x == 0) {
        atomicOr(&g_gemm_status, 1u);
        // give MMAs still in flight a bounded time to retire before the memory is freed
        if (issued > 0) mbar_wait(bar0 + 8 * ((issued - 1) % NSTAGE), ((issued - 1) / NSTAGE) & 1);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN) : "memory");
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

// loss of one minibatch: the rows' squared errors summed in FP64 in a fixed
// order (thread-strided, then a shared-memory tree), one block
__global__ void k_batch_loss(int rows, double scale, const float *rowErr, float *loss) {
    __shared__ double s[256];
    double a = 0.0;
    for (int r = threadIdx.x; r < rows; r += blockDim.x) a += rowErr[r];
    s[threadIdx.x] = a;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *loss = float(s[0] * scale);
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
    bool gemmReady[4] = {false, false, false, false};   // k_gemm forms whose shared memory limit is raised
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

// one launch of k_gemm<AT, BT> over a grid of (N / BN) x (M / BM) x parts
// tiles (the first launch of each form raises its dynamic shared memory limit)
template <bool AT, bool BT>
int gemm(ofg_mlp *m, int M, int N, int K, int kchunk, int parts, const bf16 *A, int lda, const bf16 *B, int ldb,
         float *C, int ldc, size_t zstride) {
    const int form = int(AT) * 2 + int(BT);
    if (!m->gemmReady[form]) {
        MCK(cudaFuncSetAttribute(k_gemm<AT, BT>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_GEMM));
        m->gemmReady[form] = true;
    }
    dim3 g(blocks(N, BN), blocks(M, BM), parts);
    k_gemm<AT, BT><<<g, GT, SMEM_GEMM>>>(M, N, K, kchunk, A, lda, B, ldb, C, ldc, zstride);
    return OFG_OK;
}

// after a synchronisation: an error if a GEMM wait ran out (the flag is cleared)
int gemm_status(ofg_mlp *m) {
    unsigned st = 0, zero = 0;
    MCK(cudaMemcpyFromSymbol(&st, g_gemm_status, sizeof st));
    if (st) {
        MCK(cudaMemcpyToSymbol(g_gemm_status, &zero, sizeof zero));
        return m->fail(OFG_E_TIMEOUT, "a tensor-core GEMM wait ran out");
    }
    return OFG_OK;
}

// forward through every layer for `rows` rows already packed in H[0]; with a
// target Tb, the output gradient and per-row errors as well
int forward(ofg_mlp *m, int rows, bool withTarget) {
    for (int l = 0; l < m->L; ++l) {
        int rc = gemm<false, false>(m, rows, m->N[l], m->K[l], m->K[l], 1, m->H[l], m->K[l], m->wb + m->woff[l],
                                    m->N[l], m->Z[l], m->N[l], 0);
        if (rc) return rc;
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
        int rc = gemm<true, false>(m, K, N, rows, chunk, parts, m->H[l], K, m->dZ, N, m->part, N, (size_t)K * N);
        if (rc) return rc;
        k_reduce_parts<<<blocks((int64_t)K * N, 256), 256>>>((int64_t)K * N, parts, m->part, m->gw + m->woff[l]);
        k_colsum<<<N, 256>>>(rows, N, m->dZ, m->gb + m->boff[l]);
        if (l > 0) {
            // dH = dZ W^T, then through the GELU of the layer below
            if ((rc = gemm<false, true>(m, rows, K, N, N, 1, m->dZ, N, m->wb + m->woff[l], N, m->dH, K, 0)))
                return rc;
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
        int rp = (rr + ROWS - 1) / ROWS * ROWS;
        k_pack_rows<<<blocks(rp, 128), 128>>>(rp, n, r0, m->nin, m->K[0], x, m->H[0]);
        if ((rc = forward(m, rp, false))) return rc;
        k_unpack_rows<<<blocks(rp, 128), 128>>>(rp, n, r0, m->N[m->L - 1], m->nout, m->Z[m->L - 1], y);
    }
    MCK(cudaGetLastError());
    MCK(cudaDeviceSynchronize());
    return gemm_status(m);
}

// Mean squared error of the batch X[n], Y[n] (n a multiple of 64, at most
// 65,536) and its gradient (host arrays in the parameter layout); no update
int ofg_mlp_loss_grad(ofg_mlp *m, const float *x, const float *y, int64_t n, float *loss, float *grad) {
    if (!m || !x || !y || n <= 0 || n % ROWS || n > 65536) return OFG_E_ARG;
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
    if ((rc = gemm_status(m))) return rc;
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
    if (!m || !x || !y || n <= 0 || batch <= 0 || batch % ROWS || batch > 65536 || steps < 0) return OFG_E_ARG;
    int rc = ensure_work(m, batch);
    if (rc) return rc;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    // the minibatch losses stay on the device until the end: no host
    // synchronisation between steps
    float *dLoss = nullptr;
    if (loss_out && steps > 0) MCK(cudaMalloc(&dLoss, (size_t)steps * sizeof(float)));
    for (int s = 0; s < steps; ++s) {
        k_gather<<<blocks(batch, 128), 128>>>(batch, n, m->nin, m->K[0], m->nout, x, y, seed, uint64_t(s), m->H[0],
                                              m->Tb);
        if ((rc = forward(m, batch, true)) || (rc = backward(m, batch))) {
            cudaFree(dLoss);
            return rc;
        }
        ++m->adamStep;
        float c1 = 1.0f - std::pow(b1, float(m->adamStep)), c2 = 1.0f - std::pow(b2, float(m->adamStep));
        k_adam<<<blocks(m->nw, 256), 256>>>(m->nw, m->w, m->mw, m->vw, m->gw, m->wmask, m->wb, lr, b1, b2, eps, c1, c2);
        k_adam<<<blocks(m->nb, 256), 256>>>(m->nb, m->b, m->mb, m->vb, m->gb, m->bmask, nullptr, lr, b1, b2, eps, c1,
                                            c2);
        if (dLoss) k_batch_loss<<<1, 256>>>(batch, 1.0 / (double(batch) * m->nout), m->rowErr, dLoss + s);
    }
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess && dLoss) e = cudaMemcpy(loss_out, dLoss, (size_t)steps * sizeof(float), cudaMemcpyDeviceToHost);
    cudaFree(dLoss);
    if (e != cudaSuccess) return m->fail(OFG_E_CUDA, std::string("ofg_mlp_train: ") + cudaGetErrorString(e));
    return gemm_status(m);
}

}  // extern "C"
