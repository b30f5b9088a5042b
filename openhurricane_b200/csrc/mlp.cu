// Surrogate network: BF16 tcgen05 GEMM launches, the MLP's forward and
// backward passes, Adam, and their C ABI (include/hurchem_b200.h, hc_mlp_*).
//
// Network: n_in -> L hidden layers of width H (GELU) -> n_out, trained on
// normalised inputs / outputs with a mean-squared-error loss. Parameters are
// kept in FP32 (master copy, Adam moments) and mirrored in BF16 twice: W
// [out][in] for the forward GEMM (B operand, K = in) and W^T [in][out] for
// the input-gradient GEMM (B operand, K = out). Activations are BF16,
// stored row-major (next layer's A operand) and transposed (the weight-
// gradient GEMM's B operand, K = batch). Every feature dimension is padded
// to a multiple of 64 and the batch to a multiple of 128 with zeros, which
// keep the padding rows/columns of every product zero.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <random>
#include <string>
#include <vector>

#include "../../include/hurchem_b200.h"
#include "mlp_gemm.cuh"

using namespace hc;

namespace {

}  // namespace

namespace hc {
void set_last_error(const std::string &msg);   // capi.cu: the hc_last_error() message
}  // namespace hc

namespace {

int mfail(int code, const std::string &msg) {
    hc::set_last_error(msg);
    return code;
}

#define MCUDA(call)                                                                        \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return mfail(HC_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));   \
    } while (0)

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// bf16 matrix [rows][ld] (row-major, ld elements), tile box = box_rows x 64
int make_tmap(CUtensorMap *tm, const void *base, uint64_t rows, uint64_t cols, uint64_t ld,
              uint32_t box_rows) {
    auto fn = encode_fn();
    if (!fn) return mfail(HC_E_CUDA, "cuTensorMapEncodeTiled unavailable");
    if ((reinterpret_cast<uintptr_t>(base) & 15) || (ld * 2) % 16 || cols % 64)
        return mfail(HC_E_INVALID, "GEMM operand not 16-byte aligned / padded");
    cuuint64_t dims[2] = {cols, rows};
    cuuint64_t strides[1] = {ld * 2};
    cuuint32_t box[2] = {64, box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(tm, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims,
                    strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return mfail(HC_E_CUDA, "cuTensorMapEncodeTiled failed");
    return HC_OK;
}

constexpr int kStages = 4;

template <int BN>
int launch_bn(const CUtensorMap &ta, const CUtensorMap &tb, int M, int N, int K,
              const GemmEpilogue &ep, int *err, cudaStream_t st) {
    auto kern = gemm_bf16_tn_kernel<BN, kStages>;
    const size_t smem = (size_t)kStages * GemmSmem<BN>::kStage + 1024 + 256;
    MCUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 grid(M / kGemmBM, N / BN);
    kern<<<grid, 128, smem, st>>>(ta, tb, K, ep, err);
    MCUDA(cudaGetLastError());
    return HC_OK;
}

}  // namespace

namespace hc {

// D[M][N] = A[M][K] * B[N][K]^T with the epilogue ep
int gemm_bf16_tn(const __nv_bfloat16 *A, int lda, const __nv_bfloat16 *B, int ldb, int M, int N,
                 int K, const GemmEpilogue &ep, int *err, cudaStream_t st) {
    if (M <= 0 || N <= 0 || K <= 0) return HC_OK;
    if (M % kGemmBM || K % kGemmBK || N % 32)
        return mfail(HC_E_INVALID, "GEMM shape must be M%128, N%32, K%64");
    const int BN = (N % 256 == 0) ? 256 : (N % 128 == 0) ? 128 : (N % 64 == 0) ? 64 : 32;
    CUtensorMap ta, tb;
    int rc = make_tmap(&ta, A, (uint64_t)M, (uint64_t)K, (uint64_t)lda, kGemmBM);
    if (rc != HC_OK) return rc;
    rc = make_tmap(&tb, B, (uint64_t)N, (uint64_t)K, (uint64_t)ldb, (uint32_t)BN);
    if (rc != HC_OK) return rc;
    switch (BN) {
    case 256: return launch_bn<256>(ta, tb, M, N, K, ep, err, st);
    case 128: return launch_bn<128>(ta, tb, M, N, K, ep, err, st);
    case 64: return launch_bn<64>(ta, tb, M, N, K, ep, err, st);
    default: return launch_bn<32>(ta, tb, M, N, K, ep, err, st);
    }
}

}  // namespace hc

// ------------------------------------------------------------------ small kernels
namespace {

__host__ __device__ inline int pad128(int x) { return (x + 127) / 128 * 128; }

// X fp32 [B][n_in] -> bf16 row-major [Bp][ldx] and (optionally) transposed
// [ldx][ldt] (zero padded)
__global__ void pack_input_kernel(const float *__restrict__ X, int B, int n_in, int Bp, int ldx,
                                  __nv_bfloat16 *__restrict__ xr, __nv_bfloat16 *__restrict__ xt,
                                  int ldt) {
    const int64_t total = (int64_t)Bp * ldx;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int b = (int)(i / ldx), j = (int)(i % ldx);
        const float v = (b < B && j < n_in) ? X[(int64_t)b * n_in + j] : 0.0f;
        const __nv_bfloat16 h = __float2bfloat16_rn(v);
        xr[i] = h;
        if (xt) xt[(int64_t)j * ldt + b] = h;
    }
}

// MSE loss on the first n_out columns of pred [Bp][ldp]; gradient dL/dpred
// = 2 (pred - y) / (B n_out) into bf16 row-major [Bp][ldg] and transposed
// [ldg][ldt]; padding rows/columns get zero. Loss partial sums are added to
// *loss (fp32 atomics, one per block).
__global__ void mse_grad_kernel(const float *__restrict__ pred, int ldp,
                                const float *__restrict__ Y, int B, int n_out, int Bp, int ldg,
                                __nv_bfloat16 *__restrict__ gr, __nv_bfloat16 *__restrict__ gt,
                                int ldt, float *__restrict__ loss) {
    __shared__ float part[32];
    float acc = 0.0f;
    const float scale = 2.0f / ((float)B * (float)n_out);
    const int64_t total = (int64_t)Bp * ldg;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int b = (int)(i / ldg), j = (int)(i % ldg);
        float g = 0.0f;
        if (b < B && j < n_out) {
            const float d = pred[(int64_t)b * ldp + j] - Y[(int64_t)b * n_out + j];
            acc += d * d;
            g = scale * d;
        }
        const __nv_bfloat16 h = __float2bfloat16_rn(g);
        gr[i] = h;
        gt[(int64_t)j * ldt + b] = h;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        float v = (threadIdx.x < (blockDim.x >> 5)) ? part[threadIdx.x] : 0.0f;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) atomicAdd(loss, v / ((float)B * (float)n_out));
    }
}

// out[r] = sum_b Gt[r][b] (bias gradient), one warp per row
__global__ void row_sum_kernel(const __nv_bfloat16 *__restrict__ Gt, int rows, int Bp, int ld,
                               float *__restrict__ out) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= rows) return;
    float s = 0.0f;
    for (int b = lane; b < Bp; b += 32) s += __bfloat162float(Gt[(int64_t)w * ld + b]);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) out[w] = s;
}

// Adam on fp32 parameters (rows x ld; only the valid block rows_v x cols_v
// is updated, padding stays zero); writes the bf16 mirrors W [rows][ld] and
// W^T [ld][rows_t]. With rows_v = 0 it only refreshes the mirrors.
__global__ void adam_kernel(float *__restrict__ w, float *__restrict__ m, float *__restrict__ v,
                            const float *__restrict__ g, int rows, int ld, int rows_v,
                            int cols_v, float lr, float b1, float b2, float eps, float c1,
                            float c2, __nv_bfloat16 *__restrict__ wb,
                            __nv_bfloat16 *__restrict__ wt, int rows_t) {
    const int64_t total = (int64_t)rows * ld;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(i / ld), c = (int)(i % ld);
        float x = w[i];
        if (r < rows_v && c < cols_v) {
            const float gi = g[i];
            const float mi = b1 * m[i] + (1.0f - b1) * gi;
            const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
            m[i] = mi;
            v[i] = vi;
            x = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
            w[i] = x;
        }
        if (wb) wb[i] = __float2bfloat16_rn(x);
        if (wt) wt[(int64_t)c * rows_t + r] = __float2bfloat16_rn(x);
    }
}

// copy fp32 pred [Bp][ldp] (first n_out columns, B rows) to Y [B][n_out]
__global__ void unpack_output_kernel(const float *__restrict__ pred, int ldp, int B, int n_out,
                                     float *__restrict__ Y) {
    const int64_t total = (int64_t)B * n_out;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int b = (int)(i / n_out), j = (int)(i % n_out);
        Y[i] = pred[(int64_t)b * ldp + j];
    }
}

inline int grid_for(int64_t n) {
    int64_t g = (n + 255) / 256;
    return (int)(g < 148 * 16 ? (g < 1 ? 1 : g) : 148 * 16);
}

}  // namespace

// ------------------------------------------------------------------ the network
struct hc_mlp_s {
    int n_in = 0, n_out = 0, n_hidden = 0, width = 0;
    int nl = 0;                       // layers = n_hidden + 1
    int cap = 0;                      // batch capacity (multiple of 128)
    std::vector<int> in, out, inp, outp;
    // parameters, per layer
    std::vector<float *> W, Wm, Wv, Wg, b, bm, bv, bg;
    std::vector<__nv_bfloat16 *> Wb, Wt;
    // activations, per layer input (nl + 1 entries: act[nl] unused)
    std::vector<__nv_bfloat16 *> act, actT, z, G, Gt;
    float *pred = nullptr;
    float *loss = nullptr;            // device scalar
    int *err = nullptr;               // device error flag of the GEMM kernels
    int64_t step = 0;
    std::vector<void *> owned;
    std::mutex mu;
};

namespace {

constexpr int kPadF = 128;            // feature dimensions pad to a multiple of 128

int padf(int x) { return (x + kPadF - 1) / kPadF * kPadF; }

template <typename T>
int dalloc(hc_mlp_t m, T **p, size_t n) {
    void *d = nullptr;
    MCUDA(cudaMalloc(&d, n * sizeof(T)));
    MCUDA(cudaMemset(d, 0, n * sizeof(T)));
    m->owned.push_back(d);
    *p = static_cast<T *>(d);
    return HC_OK;
}

#define MTRY(x)                    \
    do {                           \
        int rc_ = (x);             \
        if (rc_ != HC_OK) return rc_; \
    } while (0)

int check_err(hc_mlp_t m, cudaStream_t st) {
    int h = 0;
    MCUDA(cudaMemcpyAsync(&h, m->err, sizeof(int), cudaMemcpyDeviceToHost, st));
    MCUDA(cudaStreamSynchronize(st));
    if (h != 0) return mfail(HC_E_CUDA, "GEMM pipeline wait timed out (code " + std::to_string(h) + ")");
    return HC_OK;
}

// write the bf16 mirrors of layer l from its fp32 master copy
int mirror_layer(hc_mlp_t m, int l, cudaStream_t st) {
    const int rows = m->outp[l], ld = m->inp[l];
    adam_kernel<<<grid_for((int64_t)rows * ld), 256, 0, st>>>(
        m->W[l], m->Wm[l], m->Wv[l], m->Wg[l], rows, ld, 0, 0, 0.f, 0.f, 0.f, 1.f, 1.f, 1.f,
        m->Wb[l], m->Wt[l], rows);
    MCUDA(cudaGetLastError());
    return HC_OK;
}

}  // namespace

namespace {

// forward over a packed batch of Bp rows (act[0] filled). train: keep z and
// transposed activations for the backward pass.
int forward_packed(hc_mlp_t m, int Bp, bool train, cudaStream_t st) {
    for (int l = 0; l < m->nl; ++l) {
        GemmEpilogue ep{};
        ep.bias = m->b[l];
        if (l + 1 < m->nl) {
            ep.act = 1;
            ep.out_bf = m->act[l + 1];
            ep.ld_bf = m->inp[l + 1];
            if (train) {
                ep.z_out = m->z[l];
                ep.ld_zo = m->outp[l];
                ep.out_bt = m->actT[l + 1];
                ep.ld_bt = m->cap;
            }
        } else {
            ep.out_f32 = m->pred;
            ep.ld_f32 = m->outp[l];
        }
        MTRY(gemm_bf16_tn(m->act[l], m->inp[l], m->Wb[l], m->inp[l], Bp, m->outp[l], m->inp[l],
                          ep, m->err, st));
    }
    return HC_OK;
}

// gradients of the loss of (X, Y) into Wg / bg; loss added to m->loss
int backward_batch(hc_mlp_t m, const float *X, const float *Y, int B, cudaStream_t st) {
    if (B <= 0 || B > m->cap) return mfail(HC_E_INVALID, "batch exceeds the network's capacity");
    const int Bp = pad128(B);
    // transposed activations use the capacity as their row stride; the
    // weight-gradient GEMMs read their first Bp columns (K = Bp)
    pack_input_kernel<<<grid_for((int64_t)Bp * m->inp[0]), 256, 0, st>>>(
        X, B, m->n_in, Bp, m->inp[0], m->act[0], m->actT[0], m->cap);
    MCUDA(cudaGetLastError());
    MTRY(forward_packed(m, Bp, true, st));
    const int L = m->nl - 1;
    mse_grad_kernel<<<grid_for((int64_t)Bp * m->outp[L]), 256, 0, st>>>(
        m->pred, m->outp[L], Y, B, m->n_out, Bp, m->outp[L], m->G[L], m->Gt[L], m->cap, m->loss);
    MCUDA(cudaGetLastError());
    for (int l = L; l >= 0; --l) {
        // dW = G^T X : A = Gt[l] [outp][Bp], B = actT[l] [inp][Bp], K = Bp
        GemmEpilogue ew{};
        ew.out_f32 = m->Wg[l];
        ew.ld_f32 = m->inp[l];
        MTRY(gemm_bf16_tn(m->Gt[l], m->cap, m->actT[l], m->cap, m->outp[l], m->inp[l], Bp, ew,
                          m->err, st));
        row_sum_kernel<<<(m->outp[l] * 32 + 255) / 256, 256, 0, st>>>(m->Gt[l], m->outp[l], Bp,
                                                                       m->cap, m->bg[l]);
        MCUDA(cudaGetLastError());
        if (l > 0) {
            // dX = G W : A = G[l] [Bp][outp], B = Wt[l] [inp][outp], K = outp; times GELU'(z)
            GemmEpilogue ex{};
            ex.gate_z = m->z[l - 1];
            ex.ld_gz = m->outp[l - 1];
            ex.out_bf = m->G[l - 1];
            ex.ld_bf = m->outp[l - 1];
            ex.out_bt = m->Gt[l - 1];
            ex.ld_bt = m->cap;
            MTRY(gemm_bf16_tn(m->G[l], m->outp[l], m->Wt[l], m->outp[l], Bp, m->inp[l],
                              m->outp[l], ex, m->err, st));
        }
    }
    return HC_OK;
}

}  // namespace

extern "C" {

int hc_mlp_create(int n_in, int n_out, int n_hidden, int width, int max_batch, uint64_t seed,
                  hc_mlp_t *out) {
    if (!out) return mfail(HC_E_INVALID, "null output handle");
    *out = nullptr;
    if (n_in <= 0 || n_out <= 0 || n_hidden < 1 || width <= 0 || max_batch <= 0)
        return mfail(HC_E_INVALID, "bad network shape");
    if (n_in > 1024 || n_out > 1024 || width > 1024 || n_hidden > 16)
        return mfail(HC_E_INVALID, "network too large (features <= 1024, hidden layers <= 16)");
    hc_mlp_t m = new hc_mlp_s();
    m->n_in = n_in;
    m->n_out = n_out;
    m->n_hidden = n_hidden;
    m->width = width;
    m->nl = n_hidden + 1;
    m->cap = pad128(max_batch);
    for (int l = 0; l < m->nl; ++l) {
        const int i = (l == 0) ? n_in : width;
        const int o = (l + 1 == m->nl) ? n_out : width;
        m->in.push_back(i);
        m->out.push_back(o);
        m->inp.push_back(padf(i));
        m->outp.push_back(padf(o));
    }
    const int L = m->nl;
    m->W.resize(L); m->Wm.resize(L); m->Wv.resize(L); m->Wg.resize(L);
    m->b.resize(L); m->bm.resize(L); m->bv.resize(L); m->bg.resize(L);
    m->Wb.resize(L); m->Wt.resize(L);
    m->act.resize(L); m->actT.resize(L); m->z.resize(L); m->G.resize(L); m->Gt.resize(L);
    auto cleanup = [&](int rc) {
        hc_mlp_destroy(m);
        return rc;
    };
    std::mt19937_64 rng(seed);
    for (int l = 0; l < L; ++l) {
        const size_t nw = (size_t)m->outp[l] * m->inp[l];
        int rc = HC_OK;
        if ((rc = dalloc(m, &m->W[l], nw)) || (rc = dalloc(m, &m->Wm[l], nw)) ||
            (rc = dalloc(m, &m->Wv[l], nw)) || (rc = dalloc(m, &m->Wg[l], nw)) ||
            (rc = dalloc(m, &m->b[l], (size_t)m->outp[l])) ||
            (rc = dalloc(m, &m->bm[l], (size_t)m->outp[l])) ||
            (rc = dalloc(m, &m->bv[l], (size_t)m->outp[l])) ||
            (rc = dalloc(m, &m->bg[l], (size_t)m->outp[l])) || (rc = dalloc(m, &m->Wb[l], nw)) ||
            (rc = dalloc(m, &m->Wt[l], nw)) ||
            (rc = dalloc(m, &m->act[l], (size_t)m->cap * m->inp[l])) ||
            (rc = dalloc(m, &m->actT[l], (size_t)m->cap * m->inp[l])) ||
            (rc = dalloc(m, &m->G[l], (size_t)m->cap * m->outp[l])) ||
            (rc = dalloc(m, &m->Gt[l], (size_t)m->cap * m->outp[l])))
            return cleanup(rc);
        if (l + 1 < L && (rc = dalloc(m, &m->z[l], (size_t)m->cap * m->outp[l])))
            return cleanup(rc);
        // U(-1/sqrt(in), 1/sqrt(in)) for weights and biases
        const float bound = 1.0f / std::sqrt((float)m->in[l]);
        std::uniform_real_distribution<float> U(-bound, bound);
        std::vector<float> hw(nw, 0.0f), hb((size_t)m->outp[l], 0.0f);
        for (int o = 0; o < m->out[l]; ++o)
            for (int i = 0; i < m->in[l]; ++i) hw[(size_t)o * m->inp[l] + i] = U(rng);
        for (int o = 0; o < m->out[l]; ++o) hb[o] = U(rng);
        if (cudaMemcpy(m->W[l], hw.data(), nw * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(m->b[l], hb.data(), hb.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess)
            return cleanup(mfail(HC_E_CUDA, "parameter upload failed"));
        if ((rc = mirror_layer(m, l, nullptr))) return cleanup(rc);
    }
    int rc = HC_OK;
    if ((rc = dalloc(m, &m->pred, (size_t)m->cap * m->outp[L - 1])) ||
        (rc = dalloc(m, &m->loss, 1)) || (rc = dalloc(m, &m->err, 1)))
        return cleanup(rc);
    if (cudaDeviceSynchronize() != cudaSuccess) return cleanup(mfail(HC_E_CUDA, "init failed"));
    *out = m;
    return HC_OK;
}

int hc_mlp_destroy(hc_mlp_t m) {
    if (!m) return HC_OK;
    for (void *p : m->owned) cudaFree(p);
    delete m;
    return HC_OK;
}

int64_t hc_mlp_num_params(hc_mlp_t m) {
    if (!m) return -1;
    int64_t n = 0;
    for (int l = 0; l < m->nl; ++l) n += (int64_t)m->out[l] * m->in[l] + m->out[l];
    return n;
}

// host layout, layer by layer: W [out][in] row-major, then b [out]
int hc_mlp_get_params(hc_mlp_t m, float *host) {
    if (!m || !host) return mfail(HC_E_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(m->mu);
    MCUDA(cudaDeviceSynchronize());
    size_t off = 0;
    for (int l = 0; l < m->nl; ++l) {
        MCUDA(cudaMemcpy2D(host + off, sizeof(float) * m->in[l], m->W[l], sizeof(float) * m->inp[l],
                           sizeof(float) * m->in[l], m->out[l], cudaMemcpyDeviceToHost));
        off += (size_t)m->out[l] * m->in[l];
        MCUDA(cudaMemcpy(host + off, m->b[l], sizeof(float) * m->out[l], cudaMemcpyDeviceToHost));
        off += m->out[l];
    }
    return HC_OK;
}

int hc_mlp_set_params(hc_mlp_t m, const float *host) {
    if (!m || !host) return mfail(HC_E_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(m->mu);
    MCUDA(cudaDeviceSynchronize());
    size_t off = 0;
    for (int l = 0; l < m->nl; ++l) {
        MCUDA(cudaMemcpy2D(m->W[l], sizeof(float) * m->inp[l], host + off, sizeof(float) * m->in[l],
                           sizeof(float) * m->in[l], m->out[l], cudaMemcpyHostToDevice));
        off += (size_t)m->out[l] * m->in[l];
        MCUDA(cudaMemcpy(m->b[l], host + off, sizeof(float) * m->out[l], cudaMemcpyHostToDevice));
        off += m->out[l];
        MTRY(mirror_layer(m, l, nullptr));
    }
    MCUDA(cudaDeviceSynchronize());
    return HC_OK;
}

}  // extern "C"

extern "C" {

// gradients of the mean-squared error of (X, Y) (device fp32, [B][n_in] /
// [B][n_out]) w.r.t. every parameter, copied to grad_host in the parameter
// layout; loss_host (optional) receives the loss. Synchronises the stream.
int hc_mlp_grad(hc_mlp_t m, const float *X, const float *Y, int B, float *grad_host,
                float *loss_host, void *stream) {
    if (!m || !X || !Y) return mfail(HC_E_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(m->mu);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    MCUDA(cudaMemsetAsync(m->err, 0, sizeof(int), st));
    MCUDA(cudaMemsetAsync(m->loss, 0, sizeof(float), st));
    MTRY(backward_batch(m, X, Y, B, st));
    MTRY(check_err(m, st));
    if (loss_host) MCUDA(cudaMemcpy(loss_host, m->loss, sizeof(float), cudaMemcpyDeviceToHost));
    if (grad_host) {
        size_t off = 0;
        for (int l = 0; l < m->nl; ++l) {
            MCUDA(cudaMemcpy2D(grad_host + off, sizeof(float) * m->in[l], m->Wg[l],
                               sizeof(float) * m->inp[l], sizeof(float) * m->in[l], m->out[l],
                               cudaMemcpyDeviceToHost));
            off += (size_t)m->out[l] * m->in[l];
            MCUDA(cudaMemcpy(grad_host + off, m->bg[l], sizeof(float) * m->out[l],
                             cudaMemcpyDeviceToHost));
            off += m->out[l];
        }
    }
    return HC_OK;
}

// one Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on the batch (X, Y);
// stream-ordered. loss_host (optional) receives the batch loss and makes the
// call synchronous; so does check != 0, which also reads the GEMM error flag.
int hc_mlp_train_step(hc_mlp_t m, const float *X, const float *Y, int B, float lr,
                      float *loss_host, int check, void *stream) {
    if (!m || !X || !Y) return mfail(HC_E_INVALID, "null argument");
    if (!(lr > 0.0f)) return mfail(HC_E_INVALID, "learning rate must be positive");
    std::lock_guard<std::mutex> lk(m->mu);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    MCUDA(cudaMemsetAsync(m->loss, 0, sizeof(float), st));
    MTRY(backward_batch(m, X, Y, B, st));
    m->step += 1;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float c1 = 1.0f - std::pow(b1, (float)m->step), c2 = 1.0f - std::pow(b2, (float)m->step);
    for (int l = 0; l < m->nl; ++l) {
        const int rows = m->outp[l], ld = m->inp[l];
        adam_kernel<<<grid_for((int64_t)rows * ld), 256, 0, st>>>(
            m->W[l], m->Wm[l], m->Wv[l], m->Wg[l], rows, ld, m->out[l], m->in[l], lr, b1, b2, eps,
            c1, c2, m->Wb[l], m->Wt[l], rows);
        adam_kernel<<<grid_for(rows), 256, 0, st>>>(m->b[l], m->bm[l], m->bv[l], m->bg[l], 1, rows,
                                                    1, m->out[l], lr, b1, b2, eps, c1, c2, nullptr,
                                                    nullptr, 1);
        MCUDA(cudaGetLastError());
    }
    if (check) MTRY(check_err(m, st));
    if (loss_host) {
        MCUDA(cudaMemcpyAsync(loss_host, m->loss, sizeof(float), cudaMemcpyDeviceToHost, st));
        MCUDA(cudaStreamSynchronize(st));
    }
    return HC_OK;
}

// Y[B][n_out] = net(X[B][n_in]) (device fp32), in chunks of the capacity
int hc_mlp_forward(hc_mlp_t m, const float *X, int64_t B, float *Y, void *stream) {
    if (!m || !X || !Y) return mfail(HC_E_INVALID, "null argument");
    if (B <= 0) return HC_OK;
    std::lock_guard<std::mutex> lk(m->mu);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    for (int64_t r0 = 0; r0 < B; r0 += m->cap) {
        const int nb = (int)std::min<int64_t>(m->cap, B - r0);
        const int Bp = pad128(nb);
        pack_input_kernel<<<grid_for((int64_t)Bp * m->inp[0]), 256, 0, st>>>(
            X + r0 * m->n_in, nb, m->n_in, Bp, m->inp[0], m->act[0], nullptr, 0);
        MCUDA(cudaGetLastError());
        MTRY(forward_packed(m, Bp, false, st));
        unpack_output_kernel<<<grid_for((int64_t)nb * m->n_out), 256, 0, st>>>(
            m->pred, m->outp[m->nl - 1], nb, m->n_out, Y + r0 * m->n_out);
        MCUDA(cudaGetLastError());
    }
    return HC_OK;
}

// reads and clears the GEMM pipeline error flag (synchronises the stream)
int hc_mlp_check(hc_mlp_t m, void *stream) {
    if (!m) return mfail(HC_E_INVALID, "null argument");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int rc = check_err(m, st);
    cudaMemsetAsync(m->err, 0, sizeof(int), st);
    return rc;
}

// C = act(A B^T + bias): A [M][K], B [N][K] bf16 row-major (device), C fp32
// [M][N]; M % 128, N % 32, K % 64. Test entry for the tensor-core GEMM.
int hc_gemm_bf16_tn(const void *A, const void *B, int M, int N, int K, const float *bias,
                    int act, float *C, void *stream) {
    static int *err_dev = nullptr;
    static std::mutex emu;
    std::lock_guard<std::mutex> lk(emu);
    if (!A || !B || !C) return mfail(HC_E_INVALID, "null argument");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (!err_dev) MCUDA(cudaMalloc(&err_dev, sizeof(int)));
    MCUDA(cudaMemsetAsync(err_dev, 0, sizeof(int), st));
    GemmEpilogue ep{};
    ep.bias = bias;
    ep.act = act;
    ep.out_f32 = C;
    ep.ld_f32 = N;
    MTRY(gemm_bf16_tn(static_cast<const __nv_bfloat16 *>(A), K,
                      static_cast<const __nv_bfloat16 *>(B), K, M, N, K, ep, err_dev, st));
    int h = 0;
    MCUDA(cudaMemcpyAsync(&h, err_dev, sizeof(int), cudaMemcpyDeviceToHost, st));
    MCUDA(cudaStreamSynchronize(st));
    if (h) return mfail(HC_E_CUDA, "GEMM pipeline wait timed out");
    return HC_OK;
}

}  // extern "C"
