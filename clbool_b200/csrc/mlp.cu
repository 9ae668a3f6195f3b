// mlp.cu -- learned row sizing for the single-pass SpGEMM.
//
// A small MLP (6 -> 64 -> 64 -> 1, ReLU) predicts log2(1 + nnz) of every C row
// from six features of its A row; the learned SpGEMM gives every row a
// capacity of predicted size * margin + slack (never above the exact upper
// bound min(products, ncols)) and re-runs the rows that overflow with the
// exact two-pass form, so the result never depends on the predictor.
//
// Weights are used in BF16 (round to nearest even from FP32 master copies),
// every accumulation is FP32.  Training runs on the GPU with hand-written
// forward, backward and Adam kernels; the loss is the mean squared error in
// the (scaled) log2 space.  There is no counterpart in the reference.
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_bf16.h>

#include "spgemm.cuh"

struct clb_sizer {
    clb_controls *ctl = nullptr;
    float *params = nullptr;  // FP32 master weights (device)
    float *m = nullptr;       // Adam moments (device)
    float *v = nullptr;
    uint32_t step = 0;
};

namespace clb {

namespace {

constexpr int F = 6;    // features
constexpr int H = 64;   // hidden width
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + H * F, OFF_W2 = OFF_B1 + H, OFF_B2 = OFF_W2 + H * H,
              OFF_W3 = OFF_B2 + H, OFF_B3 = OFF_W3 + H, NPARAM = OFF_B3 + 1;
constexpr float FEAT_SCALE = 1.0f / 16.0f;  // log2 features and target are divided by 16

// BF16 weights, as the forward pass uses them, staged in shared memory.
struct SmemWeights {
    __nv_bfloat16 w1[H * F], b1[H], w2[H * H], b2[H], w3[H], b3;
};

__device__ __forceinline__ void stage_weights(const float *__restrict__ p, SmemWeights &s) {
    for (int k = threadIdx.x; k < NPARAM; k += blockDim.x) {
        const __nv_bfloat16 w = __float2bfloat16_rn(p[k]);
        if (k < OFF_B1) s.w1[k - OFF_W1] = w;
        else if (k < OFF_W2) s.b1[k - OFF_B1] = w;
        else if (k < OFF_B2) s.w2[k - OFF_W2] = w;
        else if (k < OFF_W3) s.b2[k - OFF_B2] = w;
        else if (k < OFF_B3) s.w3[k - OFF_W3] = w;
        else s.b3 = w;
    }
    __syncthreads();
}

// One row's forward pass; h1/h2 receive the post-activation values when
// non-null (training needs them for the backward pass).
// Layer 2 runs as outer products: the 64 layer-2 accumulators stay in
// registers while the layer-1 units are produced one at a time.
__device__ __forceinline__ float forward_row(const SmemWeights &s, const float (&x)[F], float *h1_out, float *h2_out) {
    float acc[H];
#pragma unroll
    for (int j = 0; j < H; ++j) acc[j] = __bfloat162float(s.b2[j]);
#pragma unroll 1
    for (int k = 0; k < H; ++k) {
        float a1 = __bfloat162float(s.b1[k]);
#pragma unroll
        for (int f = 0; f < F; ++f) a1 = fmaf(__bfloat162float(s.w1[k * F + f]), x[f], a1);
        const float h1 = fmaxf(a1, 0.0f);
        if (h1_out) h1_out[k] = h1;
#pragma unroll
        for (int j = 0; j < H; ++j) acc[j] = fmaf(__bfloat162float(s.w2[j * H + k]), h1, acc[j]);
    }
    float y = __bfloat162float(s.b3);
#pragma unroll
    for (int j = 0; j < H; ++j) {
        const float h = fmaxf(acc[j], 0.0f);
        if (h2_out) h2_out[j] = h;
        y = fmaf(__bfloat162float(s.w3[j]), h, y);
    }
    return y;
}

constexpr int MLP_NT = 128;

__global__ void __launch_bounds__(MLP_NT) predict_kernel(const float *__restrict__ params, const float *__restrict__ feat,
                                                         uint64_t n, float *__restrict__ out) {
    __shared__ SmemWeights s;
    stage_weights(params, s);
    for (uint64_t r = (uint64_t)blockIdx.x * MLP_NT + threadIdx.x; r < n; r += (uint64_t)gridDim.x * MLP_NT) {
        float x[F];
#pragma unroll
        for (int f = 0; f < F; ++f) x[f] = feat[r * F + f];
        out[r] = forward_row(s, x, nullptr, nullptr);
    }
}

// The prediction of the listed rows only: out[list[k]] for k < *count.
__global__ void __launch_bounds__(MLP_NT) predict_rows_kernel(const float *__restrict__ params,
                                                              const float *__restrict__ feat,
                                                              const uint32_t *__restrict__ list,
                                                              const uint32_t *__restrict__ count,
                                                              float *__restrict__ out) {
    __shared__ SmemWeights s;
    const uint32_t n = *count;
    if ((uint64_t)blockIdx.x * MLP_NT >= n) return;  // block-uniform: no row for this block
    stage_weights(params, s);
    for (uint32_t k = blockIdx.x * MLP_NT + threadIdx.x; k < n; k += gridDim.x * MLP_NT) {
        const uint64_t r = list[k];
        float x[F];
#pragma unroll
        for (int f = 0; f < F; ++f) x[f] = feat[r * F + f];
        out[r] = forward_row(s, x, nullptr, nullptr);
    }
}

// Training forward + output gradient: stores h1, h2 and dy = 2 (y - t) / n.
__global__ void __launch_bounds__(MLP_NT) train_forward_kernel(const float *__restrict__ params,
                                                               const float *__restrict__ feat,
                                                               const float *__restrict__ target, uint64_t n,
                                                               float *__restrict__ h1, float *__restrict__ h2,
                                                               float *__restrict__ dy, float *__restrict__ loss) {
    __shared__ SmemWeights s;
    __shared__ float red[MLP_NT / 32];
    stage_weights(params, s);
    float mine = 0.f;
    for (uint64_t r = (uint64_t)blockIdx.x * MLP_NT + threadIdx.x; r < n; r += (uint64_t)gridDim.x * MLP_NT) {
        float x[F];
#pragma unroll
        for (int f = 0; f < F; ++f) x[f] = feat[r * F + f];
        const float y = forward_row(s, x, h1 + r * H, h2 + r * H);
        const float e = y - target[r];
        dy[r] = 2.0f * e / (float)n;
        mine += e * e;
    }
    mine = warp_sum(mine);
    if (lane_id() == 0) red[warp_id()] = mine;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int w = 0; w < MLP_NT / 32; ++w) t += red[w];
        atomicAdd(loss, t / (float)n);
    }
}

// Per-row backward: dh2 = dy * w3 * [h2 > 0]; dh1 = W2^T dh2 * [h1 > 0].
__global__ void __launch_bounds__(MLP_NT) train_backward_rows_kernel(const float *__restrict__ params,
                                                                     const float *__restrict__ h1,
                                                                     const float *__restrict__ h2,
                                                                     const float *__restrict__ dy, uint64_t n,
                                                                     float *__restrict__ dh1, float *__restrict__ dh2) {
    __shared__ SmemWeights s;
    stage_weights(params, s);
    for (uint64_t r = (uint64_t)blockIdx.x * MLP_NT + threadIdx.x; r < n; r += (uint64_t)gridDim.x * MLP_NT) {
        const float d = dy[r];
        float g2[H];
#pragma unroll
        for (int j = 0; j < H; ++j) {
            g2[j] = h2[r * H + j] > 0.f ? d * __bfloat162float(s.w3[j]) : 0.f;
            dh2[r * H + j] = g2[j];
        }
        for (int k = 0; k < H; ++k) {
            float acc = 0.f;
#pragma unroll
            for (int j = 0; j < H; ++j) acc = fmaf(__bfloat162float(s.w2[j * H + k]), g2[j], acc);
            dh1[r * H + k] = h1[r * H + k] > 0.f ? acc : 0.f;
        }
    }
}

// Weight gradients: every thread owns parameter entries and sums their
// per-row contributions over a slice of `rps` rows, then adds the slice total
// into grad (FP32 atomics).  Slice = blockIdx.y.
constexpr int GRAD_NT = 256;
constexpr uint64_t GRAD_ROWS_PER_SLICE = 512;
constexpr uint64_t GRAD_MAX_SLICES = 65535;  // gridDim.y limit

__global__ void __launch_bounds__(GRAD_NT) train_weight_grads_kernel(const float *__restrict__ feat,
                                                                     const float *__restrict__ h1,
                                                                     const float *__restrict__ h2,
                                                                     const float *__restrict__ dy,
                                                                     const float *__restrict__ dh1,
                                                                     const float *__restrict__ dh2, uint64_t n,
                                                                     uint64_t rps, float *__restrict__ grad) {
    const uint64_t r0 = (uint64_t)blockIdx.y * rps;
    const uint64_t r1 = min(n, r0 + rps);
    for (int p = blockIdx.x * GRAD_NT + threadIdx.x; p < NPARAM; p += gridDim.x * GRAD_NT) {
        float acc = 0.f;
        if (p < OFF_B1) {  // W1[j][f] += dh1[j] x[f]
            const int j = (p - OFF_W1) / F, f = (p - OFF_W1) % F;
            for (uint64_t r = r0; r < r1; ++r) acc = fmaf(dh1[r * H + j], feat[r * F + f], acc);
        } else if (p < OFF_W2) {
            const int j = p - OFF_B1;
            for (uint64_t r = r0; r < r1; ++r) acc += dh1[r * H + j];
        } else if (p < OFF_B2) {  // W2[j][k] += dh2[j] h1[k]
            const int j = (p - OFF_W2) / H, k = (p - OFF_W2) % H;
            for (uint64_t r = r0; r < r1; ++r) acc = fmaf(dh2[r * H + j], h1[r * H + k], acc);
        } else if (p < OFF_W3) {
            const int j = p - OFF_B2;
            for (uint64_t r = r0; r < r1; ++r) acc += dh2[r * H + j];
        } else if (p < OFF_B3) {  // W3[j] += dy h2[j]
            const int j = p - OFF_W3;
            for (uint64_t r = r0; r < r1; ++r) acc = fmaf(dy[r], h2[r * H + j], acc);
        } else {
            for (uint64_t r = r0; r < r1; ++r) acc += dy[r];
        }
        atomicAdd(grad + p, acc);
    }
}

__global__ void adam_kernel(float *__restrict__ params, float *__restrict__ m, float *__restrict__ v,
                            const float *__restrict__ grad, float lr, float b1, float b2, float eps, float c1,
                            float c2) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < NPARAM; p += gridDim.x * blockDim.x) {
        const float g = grad[p];
        const float mm = b1 * m[p] + (1.f - b1) * g;
        const float vv = b2 * v[p] + (1.f - b2) * g * g;
        m[p] = mm;
        v[p] = vv;
        params[p] -= lr * (mm / c1) / (sqrtf(vv / c2) + eps);
    }
}

// Six features of every A row of A*B, plus its products (the workload):
//   log2(1+|A_i|), log2(1+P_i), log2(1+max |B_k|), log2(1+min |B_k|) (k with
//   |B_k| > 0; 0 if none), A.rows[i] / A.nrows, log2(B.nrows * B.ncols / nnz(B));
// the log2 features are scaled by 1/16.
constexpr int FT_NT = 256, FT_GROUP = 8;
constexpr uint32_t FT_LONG = 256;  // rows with more A entries: one CTA each

// Rows to size by prediction (RowSel::above > 0): only rows with more than
// `above` products get their features written, and are listed in list[0,
// *count) for the prediction; the others only get their products.
struct RowSel {
    uint32_t above = 0;
    uint32_t *list = nullptr;
    uint32_t *count = nullptr;
};

__device__ __forceinline__ void write_features(float *__restrict__ feat, uint32_t *__restrict__ work, uint64_t row,
                                               uint64_t len, uint32_t s, uint32_t mx, uint32_t mn, float rowpos,
                                               float density_term, const RowSel &sel) {
    if (work) work[row] = s;
    if (sel.above) {
        if (s <= sel.above) return;
        sel.list[atomicAdd(sel.count, 1u)] = (uint32_t)row;
    }
    if (mn == 0xFFFFFFFFu) mn = 0;
    float *f = feat + row * F;
    f[0] = log2f(1.0f + (float)len) * FEAT_SCALE;
    f[1] = log2f(1.0f + (float)s) * FEAT_SCALE;
    f[2] = log2f(1.0f + (float)mx) * FEAT_SCALE;
    f[3] = log2f(1.0f + (float)mn) * FEAT_SCALE;
    f[4] = rowpos;
    f[5] = density_term;
}

// Row position and density features of A row `row`: relative to A itself,
// or, in a stacked batch (br.row_pair non-null), to the row's own pair.
__device__ __forceinline__ void row_context(const AView &a, uint64_t row, uint64_t a_nrows, float density_term,
                                            const BatchRows &br, float &rowpos, float &dens) {
    if (br.row_pair) {
        const PairFeat p = br.pairs[br.row_pair[row]];
        rowpos = p.nrows ? (float)((double)(a.rows[row] - p.row0) / (double)p.nrows) : 0.0f;
        dens = p.density;
    } else {
        rowpos = a_nrows ? (float)((double)a.rows[row] / (double)a_nrows) : 0.0f;
        dens = density_term;
    }
}

// A group of 8 lanes per A row; rows over FT_LONG entries are listed for
// features_long_kernel (hub rows would keep 8 lanes busy long after the rest).
__global__ void __launch_bounds__(FT_NT) features_kernel(AView a, BRows b, uint64_t a_nrows, float density_term,
                                                         BatchRows br, RowSel sel, float *__restrict__ feat,
                                                         uint32_t *__restrict__ work,
                                                         uint32_t *__restrict__ long_rows,
                                                         uint32_t *__restrict__ n_long) {
    const uint32_t gl = threadIdx.x & (FT_GROUP - 1);
    const uint32_t gmask = 0xFFu << (lane_id() & 24u);
    for (uint64_t row = ((uint64_t)blockIdx.x * FT_NT + threadIdx.x) / FT_GROUP; row < a.nzr;
         row += (uint64_t)gridDim.x * (FT_NT / FT_GROUP)) {
        const uint64_t ja = a.rpt[row], je = a.rpt[row + 1];
        if (je - ja > FT_LONG) {  // the whole group takes this branch
            if (gl == 0) long_rows[atomicAdd(n_long, 1u)] = (uint32_t)row;
            continue;
        }
        uint32_t s = 0, mx = 0, mn = 0xFFFFFFFFu;
        for (uint64_t j = ja + gl; j < je; j += FT_GROUP) {
            uint64_t bb;
            const uint32_t len = b_row(b, __ldg(a.cols + j), bb);
            s += len;
            mx = max(mx, len);
            if (len) mn = min(mn, len);
        }
#pragma unroll
        for (int d = FT_GROUP / 2; d > 0; d >>= 1) {
            s += __shfl_xor_sync(gmask, s, d);
            mx = max(mx, __shfl_xor_sync(gmask, mx, d));
            mn = min(mn, __shfl_xor_sync(gmask, mn, d));
        }
        if (gl == 0) {
            float rowpos, dens;
            row_context(a, row, a_nrows, density_term, br, rowpos, dens);
            write_features(feat, work, row, je - ja, s, mx, mn, rowpos, dens, sel);
        }
    }
}

// The listed long rows, one CTA per row.
__global__ void __launch_bounds__(FT_NT) features_long_kernel(AView a, BRows b, uint64_t a_nrows, float density_term,
                                                              BatchRows br, RowSel sel,
                                                              const uint32_t *__restrict__ long_rows,
                                                              const uint32_t *__restrict__ n_long,
                                                              float *__restrict__ feat, uint32_t *__restrict__ work) {
    __shared__ uint32_t red[3][FT_NT / 32];
    const uint32_t n = *n_long;
    for (uint32_t i = blockIdx.x; i < n; i += gridDim.x) {
        const uint32_t row = long_rows[i];
        const uint64_t ja = a.rpt[row], je = a.rpt[row + 1];
        uint32_t s = 0, mx = 0, mn = 0xFFFFFFFFu;
#pragma unroll 4
        for (uint64_t j = ja + threadIdx.x; j < je; j += FT_NT) {
            uint64_t bb;
            const uint32_t len = b_row(b, __ldg(a.cols + j), bb);
            s += len;
            mx = max(mx, len);
            if (len) mn = min(mn, len);
        }
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) {
            s += __shfl_xor_sync(0xFFFFFFFFu, s, d);
            mx = max(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, d));
            mn = min(mn, __shfl_xor_sync(0xFFFFFFFFu, mn, d));
        }
        if (lane_id() == 0) {
            red[0][warp_id()] = s;
            red[1][warp_id()] = mx;
            red[2][warp_id()] = mn;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int w = 1; w < FT_NT / 32; ++w) {
                s += red[0][w];
                mx = max(mx, red[1][w]);
                mn = min(mn, red[2][w]);
            }
            float rowpos, dens;
            row_context(a, row, a_nrows, density_term, br, rowpos, dens);
            write_features(feat, work, row, je - ja, s, mx, mn, rowpos, dens, sel);
        }
        __syncthreads();
    }
}

// capacity = clamp(ceil((2^(16 y + margin) - 1) + slack), 1, min(P, ncols)) for
// the bitmap rows (more than `exact_below` products); the lighter rows get
// their exact bound min(P, ncols): they hold a small share of the products,
// and the ESC accumulators that serve them need no capacity check.
// row_ncols (may be null): per row, the columns of its product (a stacked
// batch of pairs).  defer: a single-chunk bitmap row of at least
// BMP_DEFER_MIN_WORDS words whose capacity reaches 1 / BMP_DEFER_DIV of its
// bitmap's words gets at least the bitmap's words, so that it can keep its
// bitmap in the slot.
__global__ void capacity_kernel(const float *__restrict__ pred, const uint32_t *__restrict__ work, uint64_t n,
                                uint64_t ncols, const uint32_t *__restrict__ row_ncols, float margin_log2, float slack,
                                uint32_t exact_below, bool defer, uint32_t *__restrict__ cap) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t ub = min((uint64_t)work[i], row_ncols ? (uint64_t)row_ncols[i] : ncols);
        if (work[i] <= exact_below) {
            cap[i] = (uint32_t)ub;
            continue;
        }
        const float e = pred[i] / FEAT_SCALE + margin_log2;
        const float c = exp2f(fminf(e, 40.0f)) - 1.0f + slack;
        uint64_t k = c <= 1.0f ? 1 : (c >= 4.0e9f ? ub : (uint64_t)ceilf(c));
        if (k > ub) k = ub;
        if (ub == 0) k = 0;
        if (defer) {
            const uint64_t rn = row_ncols ? (uint64_t)row_ncols[i] : ncols;
            const uint32_t wr = bitmap_words(rn);
            if (wr >= BMP_DEFER_MIN_WORDS && rn <= (uint64_t)wr * 32 && k * BMP_DEFER_DIV >= wr && k < wr) k = wr;
        }
        cap[i] = (uint32_t)k;
    }
}

unsigned grid_for(const clb_controls *ctl, uint64_t n, int nt = 256, int per_sm = 8) {
    uint64_t g = (n + nt - 1) / nt, c = (uint64_t)ctl->sm_count * per_sm;
    return (unsigned)(g > c ? c : (g ? g : 1));
}


// splitmix64: deterministic initialisation of the weights from a seed.
uint64_t splitmix(uint64_t &s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

int features_launch(clb_controls *ctl, const clb_dcsr &A, const clb_dcsr &B, const AView &a, const BRows &b,
                    float *feat, uint32_t *work, const BatchRows *batch = nullptr, const RowSel &sel = RowSel{}) {
    const BatchRows br = batch ? *batch : BatchRows{};
    Temp<uint32_t> long_rows, n_long;
    CLB_RETURN_IF(n_long.alloc(ctl, 1));
    CLB_RETURN_IF(long_rows.alloc(ctl, A.nzr ? A.nzr : 1));
    CLB_TRY_CUDA(cudaMemsetAsync(n_long.ptr, 0, 4, ctl->stream), CLB_RUN_KERNEL_FAILURE);
    ProfScope ps(ctl, "features");
    const float dt = learned_density_feature(B);
    features_kernel<<<grid_for(ctl, A.nzr * FT_GROUP), FT_NT, 0, ctl->stream>>>(a, b, A.nrows, dt, br, sel, feat,
                                                                              work, long_rows.ptr, n_long.ptr);
    features_long_kernel<<<ctl->sm_count * 4, FT_NT, 0, ctl->stream>>>(a, b, A.nrows, dt, br, sel, long_rows.ptr,
                                                                       n_long.ptr, feat, work);
    ctl->launches += 2;
    CLB_CHECK_LAUNCH();
    return CLB_SUCCESS;
}

}  // namespace

float learned_density_feature(const clb_dcsr &B) {
    if (B.nnz == 0) return 0.f;
    return (float)(std::log2((double)B.nrows * (double)B.ncols / (double)B.nnz)) * FEAT_SCALE;
}

int learned_caps(clb_controls *ctl, const clb_dcsr &A, const clb_dcsr &B, const AView &a, const BRows &b,
                 const clb_sizer *sizer, float margin_log2, float slack, const Tuning &t, const BatchRows *batch,
                 uint32_t *work, uint32_t *cap, bool defer) {
    const uint64_t n = A.nzr;
    Temp<float> feat, pred;
    Temp<uint32_t> list, count;
    CLB_RETURN_IF(feat.alloc(ctl, n * F));
    CLB_RETURN_IF(pred.alloc(ctl, n));
    CLB_RETURN_IF(list.alloc(ctl, n));
    CLB_RETURN_IF(count.alloc(ctl, 1));
    CLB_TRY_CUDA(cudaMemsetAsync(count.ptr, 0, 4, ctl->stream), CLB_RUN_KERNEL_FAILURE);
    // only the rows over t.bitmap_min products take the predicted capacity:
    // only they get features and a prediction
    RowSel sel;
    sel.above = t.bitmap_min;
    sel.list = list.ptr;
    sel.count = count.ptr;
    CLB_RETURN_IF(features_launch(ctl, A, B, a, b, feat.ptr, work, batch, sel));
    ProfScope ps(ctl, "predict");
    predict_rows_kernel<<<grid_for(ctl, n, MLP_NT, 4), MLP_NT, 0, ctl->stream>>>(sizer->params, feat.ptr, list.ptr,
                                                                                count.ptr, pred.ptr);
    capacity_kernel<<<grid_for(ctl, n), 256, 0, ctl->stream>>>(pred.ptr, work, n, B.ncols, t.row_ncols, margin_log2,
                                                              slack, t.bitmap_min, defer, cap);
    ctl->launches += 2;
    CLB_CHECK_LAUNCH();
    return CLB_SUCCESS;
}

int spgemm_learned(clb_controls *ctl, const clb_dcsr &A, const clb_dcsr &B, const clb_sizer *sizer,
                   float margin_log2, float slack, const Tuning &t, const BatchRows *batch, clb_dcsr *c,
                   clb_spgemm_stats *stats) {
    clb_spgemm_stats st{};
    ctl->launches = 0;
    if (A.nnz == 0 || B.nnz == 0 || A.nzr == 0 || B.nzr == 0) {
        clb_dcsr C{};
        C.nrows = A.nrows;
        C.ncols = B.ncols;
        *c = C;
        if (stats) *stats = st;
        return CLB_SUCCESS;
    }
    CLB_RETURN_IF(clear_status(ctl));
    const uint64_t n = A.nzr;
    const AView a{A.rpt, A.rows, A.cols, A.nzr};
    BRows b;
    Temp<uint64_t> dense, tot, wsum;
    Temp<uint32_t> work, cap;
    CLB_RETURN_IF(prepare_b(ctl, B, dense, b));
    CLB_RETURN_IF(work.alloc(ctl, n));
    CLB_RETURN_IF(cap.alloc(ctl, n));
    CLB_RETURN_IF(tot.alloc(ctl, 1));
    CLB_RETURN_IF(learned_caps(ctl, A, B, a, b, sizer, margin_log2, slack, t, batch, work.ptr, cap.ptr, true));
    // products: the single-pass driver reports them; sum the workload here
    CLB_RETURN_IF(wsum.alloc(ctl, n));
    CLB_RETURN_IF(scan_u32_to_u64(ctl, work.ptr, wsum.ptr, n, tot.ptr));
    uint64_t products = 0;
    CLB_RETURN_IF(read_scalars(ctl, tot.ptr, &products, 1));
    // ESC accumulators for the rows up to ESC_MAX_PRODUCTS products, learned
    // capacities and the spill arena (1/16 of the slots) for the bitmap rows
    int rc = spgemm_single_pass(ctl, A, B, a, b, work.ptr, cap.ptr, true, products, c, &st, 16, t);
    st.kernel_launches = ctl->launches;
    if (stats) *stats = st;
    return rc;
}

}  // namespace clb

using namespace clb;

extern "C" {

int clb_sizer_num_params(void) { return NPARAM; }

int clb_sizer_create(clb_controls *ctl, uint64_t seed, clb_sizer **out) {
    if (!ctl || !out) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    DeviceGuard g(ctl);
    *out = nullptr;
    clb_sizer *s = new clb_sizer();
    s->ctl = ctl;
    void *p = nullptr, *m = nullptr, *v = nullptr;
    if (cudaMalloc(&p, NPARAM * 4) != cudaSuccess || cudaMalloc(&m, NPARAM * 4) != cudaSuccess ||
        cudaMalloc(&v, NPARAM * 4) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(p);
        cudaFree(m);
        delete s;
        return fail(CLB_CREATE_BUFFER_ERROR, "sizer parameters");
    }
    s->params = (float *)p;
    s->m = (float *)m;
    s->v = (float *)v;
    // He-uniform initialisation for the ReLU layers, zero biases.
    std::vector<float> h(NPARAM, 0.f);
    uint64_t st = seed;
    auto uni = [&](float lim) { return (float)((splitmix(st) >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0) * lim; };
    for (int k = 0; k < H * F; ++k) h[OFF_W1 + k] = uni(std::sqrt(6.0f / F));
    for (int k = 0; k < H * H; ++k) h[OFF_W2 + k] = uni(std::sqrt(6.0f / H));
    for (int k = 0; k < H; ++k) h[OFF_W3 + k] = uni(std::sqrt(3.0f / H));
    CLB_TRY_CUDA(cudaMemcpyAsync(s->params, h.data(), NPARAM * 4, cudaMemcpyHostToDevice, ctl->stream),
                 CLB_WRITE_BUFFER_ERROR);
    CLB_TRY_CUDA(cudaStreamSynchronize(ctl->stream), CLB_EVENT_WAITING_ERROR);
    CLB_TRY_CUDA(cudaMemsetAsync(s->m, 0, NPARAM * 4, ctl->stream), CLB_RUN_KERNEL_FAILURE);
    CLB_TRY_CUDA(cudaMemsetAsync(s->v, 0, NPARAM * 4, ctl->stream), CLB_RUN_KERNEL_FAILURE);
    CLB_TRY_CUDA(cudaStreamSynchronize(ctl->stream), CLB_EVENT_WAITING_ERROR);
    *out = s;
    return CLB_SUCCESS;
}

int clb_sizer_destroy(clb_sizer *s) {
    if (!s) return CLB_SUCCESS;
    DeviceGuard g(s->ctl);
    cudaFree(s->params);
    cudaFree(s->m);
    cudaFree(s->v);
    delete s;
    return CLB_SUCCESS;
}

int clb_sizer_get_params(clb_sizer *s, float *host, size_t count) {
    if (!s || !host || count != (size_t)NPARAM) return fail(CLB_INVALID_ARGUMENT, "expected clb_sizer_num_params() floats");
    DeviceGuard g(s->ctl);
    CLB_TRY_CUDA(cudaMemcpyAsync(host, s->params, NPARAM * 4, cudaMemcpyDeviceToHost, s->ctl->stream),
                 CLB_READ_BUFFER_ERROR);
    CLB_TRY_CUDA(cudaStreamSynchronize(s->ctl->stream), CLB_EVENT_WAITING_ERROR);
    return CLB_SUCCESS;
}

int clb_sizer_set_params(clb_sizer *s, const float *host, size_t count) {
    if (!s || !host || count != (size_t)NPARAM) return fail(CLB_INVALID_ARGUMENT, "expected clb_sizer_num_params() floats");
    DeviceGuard g(s->ctl);
    CLB_TRY_CUDA(cudaMemcpyAsync(s->params, host, NPARAM * 4, cudaMemcpyHostToDevice, s->ctl->stream),
                 CLB_WRITE_BUFFER_ERROR);
    CLB_TRY_CUDA(cudaMemsetAsync(s->m, 0, NPARAM * 4, s->ctl->stream), CLB_RUN_KERNEL_FAILURE);
    CLB_TRY_CUDA(cudaMemsetAsync(s->v, 0, NPARAM * 4, s->ctl->stream), CLB_RUN_KERNEL_FAILURE);
    CLB_TRY_CUDA(cudaStreamSynchronize(s->ctl->stream), CLB_EVENT_WAITING_ERROR);
    s->step = 0;
    return CLB_SUCCESS;
}

int clb_dcsr_row_features(clb_controls *ctl, const clb_dcsr *a_, const clb_dcsr *b_, float *features,
                          uint32_t *workload) {
    if (!ctl || !a_ || !b_) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    const clb_dcsr A = *a_, B = *b_;
    CLB_RETURN_IF(validate_spgemm(A, B));
    if (A.nzr == 0) return CLB_SUCCESS;
    if (!features) return fail(CLB_INVALID_ARGUMENT, "features is NULL");
    DeviceGuard g(ctl);
    const AView a{A.rpt, A.rows, A.cols, A.nzr};
    BRows b;
    Temp<uint64_t> dense;
    CLB_RETURN_IF(prepare_b(ctl, B, dense, b));
    CLB_RETURN_IF(features_launch(ctl, A, B, a, b, features, workload));
    CLB_TRY_CUDA(cudaStreamSynchronize(ctl->stream), CLB_EVENT_WAITING_ERROR);
    return CLB_SUCCESS;
}

int clb_dcsr_row_nnz(clb_controls *ctl, const clb_dcsr *a_, const clb_dcsr *b_, uint32_t *row_nnz) {
    if (!ctl || !a_ || !b_) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    const clb_dcsr A = *a_, B = *b_;
    CLB_RETURN_IF(validate_spgemm(A, B));
    if (A.nzr == 0) return CLB_SUCCESS;
    if (!row_nnz) return fail(CLB_INVALID_ARGUMENT, "row_nnz is NULL");
    DeviceGuard g(ctl);
    CLB_TRY_CUDA(cudaMemsetAsync(row_nnz, 0, A.nzr * 4, ctl->stream), CLB_RUN_KERNEL_FAILURE);
    if (B.nnz == 0) {
        CLB_TRY_CUDA(cudaStreamSynchronize(ctl->stream), CLB_EVENT_WAITING_ERROR);
        return CLB_SUCCESS;
    }
    CLB_RETURN_IF(clear_status(ctl));
    const AView a{A.rpt, A.rows, A.cols, A.nzr};
    BRows b;
    Temp<uint64_t> dense, tot;
    Temp<uint32_t> work, list, info, flags;
    const uint64_t n = A.nzr;
    CLB_RETURN_IF(prepare_b(ctl, B, dense, b));
    CLB_RETURN_IF(tot.alloc(ctl, 1));
    CLB_RETURN_IF(work.alloc(ctl, n));
    CLB_RETURN_IF(list.alloc(ctl, n));
    CLB_RETURN_IF(info.alloc(ctl, 2 * NUM_BINS));
    CLB_RETURN_IF(flags.alloc(ctl, n));
    CLB_TRY_CUDA(cudaMemsetAsync(tot.ptr, 0, 8, ctl->stream), CLB_RUN_KERNEL_FAILURE);
    CLB_RETURN_IF(launch_workload(ctl, a, b, work.ptr, tot.ptr));
    CLB_RETURN_IF(launch_binning(ctl, work.ptr, nullptr, n, B.ncols, info.ptr, list.ptr, flags.ptr));
    BinLists bl{list.ptr, info.ptr};
    RowOut sym{row_nnz, nullptr, nullptr, nullptr, nullptr, ctl->d_status};
    sym.row_products = work.ptr;
    CLB_RETURN_IF(launch_accumulators(ctl, false, bl, a, b, sym, B.ncols, n));
    return check_status(ctl, "row_nnz");
}

int clb_sizer_predict(clb_sizer *s, const float *features, uint64_t n, float *out) {
    if (!s) return fail(CLB_INVALID_ARGUMENT, "sizer is NULL");
    if (n == 0) return CLB_SUCCESS;
    if (!features || !out) return fail(CLB_INVALID_ARGUMENT, "NULL array");
    clb_controls *ctl = s->ctl;
    DeviceGuard g(ctl);
    predict_kernel<<<grid_for(ctl, n, MLP_NT, 4), MLP_NT, 0, ctl->stream>>>(s->params, features, n, out);
    CLB_CHECK_LAUNCH();
    CLB_TRY_CUDA(cudaStreamSynchronize(ctl->stream), CLB_EVENT_WAITING_ERROR);
    return CLB_SUCCESS;
}

// Loss and gradient (w.r.t. the BF16-rounded weights) of a batch, to host.
static int batch_gradients(clb_sizer *s, const float *features, const float *targets, uint64_t n, float *d_grad,
                           float *d_loss) {
    clb_controls *ctl = s->ctl;
    Temp<float> h1, h2, dy, dh1, dh2;
    CLB_RETURN_IF(h1.alloc(ctl, n * H));
    CLB_RETURN_IF(h2.alloc(ctl, n * H));
    CLB_RETURN_IF(dy.alloc(ctl, n));
    CLB_RETURN_IF(dh1.alloc(ctl, n * H));
    CLB_RETURN_IF(dh2.alloc(ctl, n * H));
    CLB_TRY_CUDA(cudaMemsetAsync(d_grad, 0, NPARAM * 4, ctl->stream), CLB_RUN_KERNEL_FAILURE);
    CLB_TRY_CUDA(cudaMemsetAsync(d_loss, 0, 4, ctl->stream), CLB_RUN_KERNEL_FAILURE);
    train_forward_kernel<<<grid_for(ctl, n, MLP_NT, 4), MLP_NT, 0, ctl->stream>>>(s->params, features, targets, n,
                                                                                 h1.ptr, h2.ptr, dy.ptr, d_loss);
    train_backward_rows_kernel<<<grid_for(ctl, n, MLP_NT, 4), MLP_NT, 0, ctl->stream>>>(s->params, h1.ptr, h2.ptr,
                                                                                       dy.ptr, n, dh1.ptr, dh2.ptr);
    uint64_t rps = GRAD_ROWS_PER_SLICE;
    if ((n + rps - 1) / rps > GRAD_MAX_SLICES) rps = (n + GRAD_MAX_SLICES - 1) / GRAD_MAX_SLICES;
    dim3 gg((NPARAM + GRAD_NT - 1) / GRAD_NT, (unsigned)((n + rps - 1) / rps));
    train_weight_grads_kernel<<<gg, GRAD_NT, 0, ctl->stream>>>(features, h1.ptr, h2.ptr, dy.ptr, dh1.ptr, dh2.ptr, n,
                                                             rps, d_grad);
    CLB_CHECK_LAUNCH();
    return CLB_SUCCESS;
}

int clb_sizer_gradients(clb_sizer *s, const float *features, const float *targets, uint64_t n, float *grads_host,
                        float *loss_host) {
    if (!s || !features || !targets || !grads_host || n == 0) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    clb_controls *ctl = s->ctl;
    DeviceGuard g(ctl);
    Temp<float> grad, loss;
    CLB_RETURN_IF(grad.alloc(ctl, NPARAM));
    CLB_RETURN_IF(loss.alloc(ctl, 1));
    CLB_RETURN_IF(batch_gradients(s, features, targets, n, grad.ptr, loss.ptr));
    CLB_TRY_CUDA(cudaMemcpyAsync(grads_host, grad.ptr, NPARAM * 4, cudaMemcpyDeviceToHost, ctl->stream),
                 CLB_READ_BUFFER_ERROR);
    float l = 0.f;
    CLB_TRY_CUDA(cudaMemcpyAsync(&l, loss.ptr, 4, cudaMemcpyDeviceToHost, ctl->stream), CLB_READ_BUFFER_ERROR);
    CLB_TRY_CUDA(cudaStreamSynchronize(ctl->stream), CLB_EVENT_WAITING_ERROR);
    if (loss_host) *loss_host = l;
    return CLB_SUCCESS;
}

int clb_sizer_train(clb_sizer *s, const float *features, const float *targets, uint64_t n, uint32_t epochs,
                    uint32_t batch, float lr, uint64_t seed, float *final_loss) {
    if (!s || !features || !targets || n == 0 || batch == 0) return fail(CLB_INVALID_ARGUMENT, "bad argument");
    clb_controls *ctl = s->ctl;
    DeviceGuard g(ctl);
    // Mini-batches are contiguous slices of a once-shuffled copy of the data.
    std::vector<uint64_t> perm(n);
    for (uint64_t i = 0; i < n; ++i) perm[i] = i;
    uint64_t st = seed ? seed : 1;
    for (uint64_t i = n - 1; i > 0; --i) std::swap(perm[i], perm[splitmix(st) % (i + 1)]);
    std::vector<float> hf(n * F), ht(n), sf(n * F), stg(n);
    CLB_TRY_CUDA(cudaMemcpyAsync(hf.data(), features, n * F * 4, cudaMemcpyDeviceToHost, ctl->stream),
                 CLB_READ_BUFFER_ERROR);
    CLB_TRY_CUDA(cudaMemcpyAsync(ht.data(), targets, n * 4, cudaMemcpyDeviceToHost, ctl->stream),
                 CLB_READ_BUFFER_ERROR);
    CLB_TRY_CUDA(cudaStreamSynchronize(ctl->stream), CLB_EVENT_WAITING_ERROR);
    for (uint64_t i = 0; i < n; ++i) {
        memcpy(&sf[i * F], &hf[perm[i] * F], F * 4);
        stg[i] = ht[perm[i]];
    }
    Temp<float> df, dt, grad, loss;
    CLB_RETURN_IF(df.alloc(ctl, n * F));
    CLB_RETURN_IF(dt.alloc(ctl, n));
    CLB_RETURN_IF(grad.alloc(ctl, NPARAM));
    CLB_RETURN_IF(loss.alloc(ctl, 1));
    CLB_TRY_CUDA(cudaMemcpyAsync(df.ptr, sf.data(), n * F * 4, cudaMemcpyHostToDevice, ctl->stream),
                 CLB_WRITE_BUFFER_ERROR);
    CLB_TRY_CUDA(cudaMemcpyAsync(dt.ptr, stg.data(), n * 4, cudaMemcpyHostToDevice, ctl->stream),
                 CLB_WRITE_BUFFER_ERROR);
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    float last = 0.f;
    for (uint32_t ep = 0; ep < epochs; ++ep) {
        for (uint64_t o = 0; o < n; o += batch) {
            const uint64_t m = min((uint64_t)batch, n - o);
            CLB_RETURN_IF(batch_gradients(s, df.ptr + o * F, dt.ptr + o, m, grad.ptr, loss.ptr));
            ++s->step;
            const float c1 = 1.f - powf(b1, (float)s->step), c2 = 1.f - powf(b2, (float)s->step);
            adam_kernel<<<(NPARAM + 255) / 256, 256, 0, ctl->stream>>>(s->params, s->m, s->v, grad.ptr, lr, b1, b2,
                                                                       eps, c1, c2);
            CLB_CHECK_LAUNCH();
        }
        CLB_TRY_CUDA(cudaMemcpyAsync(&last, loss.ptr, 4, cudaMemcpyDeviceToHost, ctl->stream), CLB_READ_BUFFER_ERROR);
    }
    CLB_TRY_CUDA(cudaStreamSynchronize(ctl->stream), CLB_EVENT_WAITING_ERROR);
    if (final_loss) *final_loss = last;
    return CLB_SUCCESS;
}

int clb_dcsr_spgemm_learned(clb_controls *ctl, const clb_dcsr *a_, const clb_dcsr *b_, const clb_sizer *sizer,
                            float margin_log2, float slack, const clb_spgemm_tuning *tuning, clb_dcsr *c,
                            clb_spgemm_stats *stats) {
    if (!ctl || !a_ || !b_ || !c || !sizer) return fail(CLB_INVALID_ARGUMENT, "NULL argument");
    CLB_RETURN_IF(check_tuning(tuning));
    CLB_RETURN_IF(validate_spgemm(*a_, *b_));
    DeviceGuard g(ctl);
    return spgemm_learned(ctl, *a_, *b_, sizer, margin_log2, slack, to_tuning(tuning), nullptr, c, stats);
}

}  // extern "C"
