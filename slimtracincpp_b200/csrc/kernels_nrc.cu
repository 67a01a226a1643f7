// Radiance-cache MLP kernels on the sm_100a tensor cores (tcgen05).
//
// One CTA of 128 threads owns a tile of 128 samples; thread t is sample row t,
// which is also TMEM lane t of the M=128 accumulators.  Per layer one elected
// thread issues the tcgen05.mma chain (K=16 per instruction) and commits it
// to an mbarrier; every thread waits, reads its accumulator row with
// tcgen05.ld, applies the activation and writes its bf16 row into the next
// operand image in shared memory.
//
//   infer  forward only; 80 KB of shared memory, 128 TMEM columns, persistent
//          over tiles (grid = 2 CTAs per SM).
//   train  forward, log-radiance L2 output gradient, backward; 162 KB of shared
//          memory (weights, the input tile, the four hidden tiles, two
//          gradient tiles), 512 TMEM columns: the forward and input-gradient
//          accumulators plus one accumulator per weight matrix that sums
//          dW over every tile the CTA processes.  Each CTA writes its dW sums
//          to its own row of a partial buffer; the Adam kernel adds the rows
//          in a fixed order (deterministic) and updates the f32 master
//          weights, the moments and the bf16 image.
//
// GEMMs per 128-sample tile (M x N x K):
//   forward   H1 = X W0^T 128x64x96, H2..H4 128x64x64, z = H4 W4^T 128x16x64
//   backward  dW4^T += H4^T g4   64x16x128   dH4 = g4 W4   128x64x16
//             dW_l  += g_l^T H_l 64x64x128   dH_l = g_l W_l 128x64x64 (l = 3..1)
//             dW0   += g0^T X    64x96x128
// The weight-gradient GEMMs read the sample-major activation and gradient
// tiles MN-major (rows = samples = K); the input-gradient GEMMs read the
// weight images MN-major.
#include <cuda_bf16.h>

#include "nrc.h"
#include "umma.cuh"

namespace slim {
namespace nrc {

using namespace umma;

#define SLIM_N __device__ __forceinline__

constexpr uint32_t kXBytes = kTile * kInputs * 2;    // 24576
constexpr uint32_t kHBytes = kTile * kHidden * 2;    // 16384
constexpr uint32_t kGBytes = kTile * kOutPad * 2;    // 4096 (output gradient tile)
constexpr uint32_t kInferSmem = kImgBytes + kXBytes + kHBytes;                       // 79872
constexpr uint32_t kTrainSmem = kImgBytes + kXBytes + 4 * kHBytes + 2 * kHBytes + kGBytes;   // 165888

// TMEM columns
constexpr uint32_t kColFwd = 0, kColOut = 64, kColDH = 128;
constexpr uint32_t kColDW0 = 192, kColDW1 = 288, kColDW4 = 480;   // dW1..dW3 at 288, 352, 416

constexpr uint32_t kIdHidden0 = idesc_bf16(128, 64, 0, 0);
constexpr uint32_t kIdOut = idesc_bf16(128, 16, 0, 0);
constexpr uint32_t kIdDH = idesc_bf16(128, 64, 0, 1);    // g (K-major) x W (MN-major)
constexpr uint32_t kIdDW = idesc_bf16(64, 64, 1, 1);
constexpr uint32_t kIdDW0 = idesc_bf16(64, 96, 1, 1);
constexpr uint32_t kIdDW4 = idesc_bf16(64, 16, 1, 1);

SLIM_N uint32_t img_off(uint32_t rows, uint32_t r, uint32_t c) {
    return (c >> 3) * (rows * 16u) + (r >> 3) * 128u + (r & 7u) * 16u + (c & 7u) * 2u;
}

SLIM_N uint32_t bf16_bits(float x) { return (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(x)); }
SLIM_N uint32_t pack2(float a, float b) { return bf16_bits(a) | (bf16_bits(b) << 16); }
SLIM_N float bf16_lo(uint32_t w) { return __uint_as_float(w << 16); }
SLIM_N float bf16_hi(uint32_t w) { return __uint_as_float(w & 0xFFFF0000u); }

// Row r, column group g (8 values) of a 128-row image.
SLIM_N void store8(uint8_t *img, uint32_t r, uint32_t g, const float v[8]) {
    uint4 q = make_uint4(pack2(v[0], v[1]), pack2(v[2], v[3]), pack2(v[4], v[5]), pack2(v[6], v[7]));
    *(uint4 *)(img + g * (kTile * 16u) + r * 16u) = q;
}
SLIM_N uint4 load8(const uint8_t *img, uint32_t r, uint32_t g) {
    return *(const uint4 *)(img + g * (kTile * 16u) + r * 16u);
}

// 32 accumulator columns of this thread's lane; the wait is part of the same
// asm statement, so no use of the values can be scheduled before it.
SLIM_N void tmem_ld32(uint32_t taddr, float v[32]) {
    uint32_t r[32];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                 "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                 "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n\t"
                 "tcgen05.wait::ld.sync.aligned;"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
                   "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
                   "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                 : "r"(taddr) : "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}
SLIM_N void tmem_ld16w(uint32_t taddr, float v[16]) {
    uint32_t r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                 "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n\t"
                 "tcgen05.wait::ld.sync.aligned;"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr) : "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// Real spherical harmonics, bands 0..3, of a unit vector.
SLIM_N void sh_bands4(float x, float y, float z, float s[16]) {
    float xx = x * x, yy = y * y, zz = z * z;
    s[0] = 0.28209479177387814f;
    s[1] = -0.48860251190291987f * y;
    s[2] = 0.48860251190291987f * z;
    s[3] = -0.48860251190291987f * x;
    s[4] = 1.0925484305920792f * x * y;
    s[5] = -1.0925484305920792f * y * z;
    s[6] = 0.94617469575755997f * zz - 0.31539156525251999f;
    s[7] = -1.0925484305920792f * x * z;
    s[8] = 0.54627421529603959f * (xx - yy);
    s[9] = -0.59004358992664352f * y * (3.0f * xx - yy);
    s[10] = 2.8906114426405538f * x * y * z;
    s[11] = 0.45704579946446572f * y * (1.0f - 5.0f * zz);
    s[12] = 0.3731763325901154f * z * (5.0f * zz - 3.0f);
    s[13] = 0.45704579946446572f * x * (1.0f - 5.0f * zz);
    s[14] = 1.4453057213202769f * z * (xx - yy);
    s[15] = 0.59004358992664352f * x * (3.0f * yy - xx);
}

// Input row of one sample (zeros for rows past the end).
SLIM_N void encode_row(const float4 *f, bool valid, uint8_t *X, uint32_t r) {
    float4 a = make_float4(0, 0, 0, 0), b = a, c = a, d = a;
    if (valid) { a = f[0]; b = f[1]; c = f[2]; d = f[3]; }
    float p[3] = {a.x, a.y, a.z};
#pragma unroll
    for (int g = 0; g < 9; g++) {
        float v[8];
#pragma unroll
        for (int j = 0; j < 8; j += 2) {
            const int col = g * 8 + j, axis = col / 24, k = (col % 24) / 2;
            float s, co;
            sincospif(p[axis] * (float)(1 << k), &s, &co);   // 2^k p is exact
            v[j] = s;
            v[j + 1] = co;
        }
        if (!valid) for (int j = 0; j < 8; j++) v[j] = 0.0f;
        store8(X, r, g, v);
    }
    float sh[16];
    sh_bands4(b.x, b.y, b.z, sh);
    if (!valid) for (int j = 0; j < 16; j++) sh[j] = 0.0f;
    store8(X, r, 9, sh);
    store8(X, r, 10, sh + 8);
    float v[8] = {c.x, c.y, c.z, a.w, d.x, d.y, d.z, valid ? 1.0f : 0.0f};
    store8(X, r, 11, v);
}

// ReLU epilogue of a hidden layer: accumulator row -> bf16 row of H.
SLIM_N void epilogue_relu(uint32_t lane_addr, uint8_t *H, uint32_t r) {
#pragma unroll
    for (int half = 0; half < 2; half++) {
        float v[32];
        tmem_ld32(lane_addr + 32u * half, v);
#pragma unroll
        for (int g = 0; g < 4; g++) {
            float w[8];
#pragma unroll
            for (int j = 0; j < 8; j++) w[j] = fmaxf(v[8 * g + j], 0.0f);
            store8(H, r, 4 * half + g, w);
        }
    }
}

// Input-gradient epilogue: g = bf16(dH * [H > 0]) for this row.
SLIM_N void epilogue_mask(uint32_t lane_addr, const uint8_t *Hact, uint8_t *G, uint32_t r) {
#pragma unroll
    for (int half = 0; half < 2; half++) {
        float v[32];
        tmem_ld32(lane_addr + 32u * half, v);
#pragma unroll
        for (int g = 0; g < 4; g++) {
            uint4 h = load8(Hact, r, 4 * half + g);
            uint32_t hw[4] = {h.x, h.y, h.z, h.w};
            float w[8];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                w[2 * j] = bf16_lo(hw[j]) > 0.0f ? v[8 * g + 2 * j] : 0.0f;
                w[2 * j + 1] = bf16_hi(hw[j]) > 0.0f ? v[8 * g + 2 * j + 1] : 0.0f;
            }
            store8(G, r, 4 * half + g, w);
        }
    }
}

// Thread-barrier step between an epilogue (generic smem writes, TMEM reads)
// and the next MMA issue.
SLIM_N void sync_for_mma() {
    fence_smem_to_async();
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
}

// ---- inference --------------------------------------------------------------
__global__ void __launch_bounds__(128) k_nrc_infer(const float4 *__restrict__ features, const uint32_t *count,
                                                   uint32_t n_host, float4 *__restrict__ radiance,
                                                   const uint8_t *__restrict__ weight_image, uint32_t *error_flags) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t *W = smem, *X = smem + kImgBytes, *H = X + kXBytes;
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_base_s;
    __shared__ int abort_s;
    const uint32_t t = threadIdx.x, warp = t >> 5;
    const uint32_t n = count ? *count : n_host;
    const uint32_t tiles = (n + kTile - 1) / kTile;
    if (blockIdx.x >= tiles) return;                       // uniform over the CTA, before any allocation
    for (uint32_t i = t; i < kImgBytes / 16; i += blockDim.x)
        ((uint4 *)W)[i] = ((const uint4 *)weight_image)[i];
    if (t == 0) { mbar_init(&bar, 1); abort_s = 0; }
    if (warp == 0) tmem_alloc(&tmem_base_s, 128);
    sync_for_mma();
    const uint32_t tb = tmem_base_s;
    const uint32_t lane = tmem_at(tb, warp * 32u, 0);
    const uint32_t sW = smem_addr(W), sX = smem_addr(X), sH = smem_addr(H);
    uint32_t phase = 0;
    bool aborted = false;
    for (uint32_t tile = blockIdx.x; tile < tiles && !aborted; tile += gridDim.x) {
        const uint32_t i = tile * kTile + t;
        const bool valid = i < n;
        encode_row(features + 4 * (size_t)i, valid, X, t);
        sync_for_mma();
        for (int l = 0; l < 5; l++) {
            if (t == 0) {
                if (l == 0) {
#pragma unroll
                    for (uint32_t k = 0; k < kInputs / 16; k++)
                        mma(tb + kColFwd, kmajor(sX, kTile, k), kmajor(sW, kHidden, k), kIdHidden0, k > 0);
                } else if (l < 4) {
                    const uint32_t w = sW + kImgOff1 + (l - 1) * kImgW;
#pragma unroll
                    for (uint32_t k = 0; k < kHidden / 16; k++)
                        mma(tb + kColFwd, kmajor(sH, kTile, k), kmajor(w, kHidden, k), kIdHidden0, k > 0);
                } else {
#pragma unroll
                    for (uint32_t k = 0; k < kHidden / 16; k++)
                        mma(tb + kColOut, kmajor(sH, kTile, k), kmajor(sW + kImgOff4, kOutPad, k), kIdOut, k > 0);
                }
                commit(&bar);
            }
            if (!mbar_wait(&bar, phase)) abort_s = 1;
            phase ^= 1u;
            fence_after_sync();
            if (l < 4) {
                epilogue_relu(lane + kColFwd, H, t);
            } else {
                float z[16];
                tmem_ld16w(lane + kColOut, z);
                if (valid)
                    radiance[i] = make_float4(fmaxf(expf(fminf(z[0], kZMax)) - kLogOffset, 0.0f),
                                              fmaxf(expf(fminf(z[1], kZMax)) - kLogOffset, 0.0f),
                                              fmaxf(expf(fminf(z[2], kZMax)) - kLogOffset, 0.0f), 0.0f);
            }
            sync_for_mma();
            if (abort_s) { aborted = true; break; }
        }
    }
    if (aborted) {
        if (t == 0) { atomicOr(error_flags, kErrTimeout); mbar_wait(&bar, phase); }
        fence_before_sync();
        __syncthreads();
    }
    if (warp == 0) tmem_free(tb, 128);
}

// ---- training -----------------------------------------------------------------
// Samples of a step: `n` from `offset` on, clipped to the device count when
// one is given (the frame's training set size is only known on the device).
SLIM_N uint32_t step_samples(uint32_t n, const uint32_t *count, uint32_t offset) {
    if (!count) return n;
    uint32_t c = *count;
    return c > offset ? (c - offset < n ? c - offset : n) : 0u;
}

__global__ void __launch_bounds__(128, 1) k_nrc_train(const float4 *__restrict__ features,
                                                      const float4 *__restrict__ targets, uint32_t n_max,
                                                      const uint32_t *count, uint32_t offset,
                                                      const uint8_t *__restrict__ weight_image,
                                                      float *__restrict__ partials, float *__restrict__ loss_partials,
                                                      uint32_t *step, uint32_t *error_flags) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t *W = smem;
    uint8_t *X = W + kImgBytes;
    uint8_t *Hs = X + kXBytes;                 // H1..H4, kHBytes each
    uint8_t *G = Hs + 4 * kHBytes;             // two gradient tiles
    uint8_t *G4 = G + 2 * kHBytes;             // output gradient tile (16 columns)
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_base_s;
    __shared__ int abort_s;
    __shared__ float loss_s[4];
    const uint32_t t = threadIdx.x, warp = t >> 5;
    const uint32_t n = step_samples(n_max, count, offset);
    const uint32_t tiles = (n + kTile - 1) / kTile;
    if (n && blockIdx.x == 0 && t == 0) atomicAdd(step, 1u);
    features += 4 * (size_t)offset;
    targets += offset;
    for (uint32_t i = t; i < kImgBytes / 16; i += blockDim.x)
        ((uint4 *)W)[i] = ((const uint4 *)weight_image)[i];
    if (t == 0) { mbar_init(&bar, 1); abort_s = 0; }
    if (warp == 0) tmem_alloc(&tmem_base_s, 512);
    sync_for_mma();
    const uint32_t tb = tmem_base_s;
    const uint32_t lane = tmem_at(tb, warp * 32u, 0);
    const uint32_t sW = smem_addr(W), sX = smem_addr(X), sH = smem_addr(Hs), sG = smem_addr(G), sG4 = smem_addr(G4);
    uint32_t phase = 0;
    bool aborted = false, first = true;
    float loss = 0.0f;

    // Wait for the MMAs committed so far; false (and the CTA stops) on timeout.
    auto wait_mma = [&]() -> bool {
        if (!mbar_wait(&bar, phase)) abort_s = 1;
        phase ^= 1u;
        fence_after_sync();
        return true;
    };

    for (uint32_t tile = blockIdx.x; tile < tiles && !aborted; tile += gridDim.x) {
        const uint32_t i = tile * kTile + t;
        const bool valid = i < n;
        encode_row(features + 4 * (size_t)i, valid, X, t);
        float4 y = valid ? targets[i] : make_float4(0, 0, 0, 0);
        sync_for_mma();
        // forward
        for (int l = 0; l < 5 && !aborted; l++) {
            if (t == 0) {
                if (l == 0) {
#pragma unroll
                    for (uint32_t k = 0; k < kInputs / 16; k++)
                        mma(tb + kColFwd, kmajor(sX, kTile, k), kmajor(sW, kHidden, k), kIdHidden0, k > 0);
                } else {
                    const uint32_t a = sH + (l - 1) * kHBytes;
                    if (l < 4) {
                        const uint32_t w = sW + kImgOff1 + (l - 1) * kImgW;
#pragma unroll
                        for (uint32_t k = 0; k < kHidden / 16; k++)
                            mma(tb + kColFwd, kmajor(a, kTile, k), kmajor(w, kHidden, k), kIdHidden0, k > 0);
                    } else {
#pragma unroll
                        for (uint32_t k = 0; k < kHidden / 16; k++)
                            mma(tb + kColOut, kmajor(a, kTile, k), kmajor(sW + kImgOff4, kOutPad, k), kIdOut, k > 0);
                    }
                }
                commit(&bar);
            }
            wait_mma();
            if (l < 4) {
                epilogue_relu(lane + kColFwd, Hs + l * kHBytes, t);
            } else {
                float z[16];
                tmem_ld16w(lane + kColOut, z);
                float dz[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                if (valid) {
                    const float tv[3] = {y.x, y.y, y.z};
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        // L2 on log radiance: z regresses log(target + offset)
                        float diff = z[c] - logf(fmaxf(tv[c], 0.0f) + kLogOffset);
                        loss += diff * diff;
                        dz[c] = 2.0f * diff;
                    }
                }
                float zero[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                store8(G4, t, 0, dz);
                store8(G4, t, 1, zero);
            }
            sync_for_mma();
            if (abort_s) aborted = true;
        }
        if (aborted) break;
        // backward: output layer
        if (t == 0) {
            mma(tb + kColDH, kmajor(sG4, kTile, 0), mnmajor(sW + kImgOff4, kOutPad, 0), kIdDH, 0);
            const uint32_t h4 = sH + 3 * kHBytes;
#pragma unroll
            for (uint32_t k = 0; k < kTile / 16; k++)
                mma(tb + kColDW4, mnmajor(h4, kTile, k), mnmajor(sG4, kTile, k), kIdDW4, (!first || k > 0));
            commit(&bar);
        }
        wait_mma();
        epilogue_mask(lane + kColDH, Hs + 3 * kHBytes, G, t);     // g3 -> G[0]
        sync_for_mma();
        if (abort_s) { aborted = true; break; }
        // hidden layers 3..1: dW_l += g_l^T H_l, dH_l = g_l W_l, g_{l-1} = mask(dH_l, H_l)
        uint32_t cur = 0;
        for (int l = 3; l >= 1; l--) {
            const uint32_t g = sG + cur * kHBytes;
            const uint32_t h = sH + (l - 1) * kHBytes;           // H_l (H1 at index 0)
            const uint32_t w = sW + kImgOff1 + (l - 1) * kImgW;  // W_l
            if (t == 0) {
                const uint32_t dcol = kColDW1 + (l - 1) * 64;
#pragma unroll
                for (uint32_t k = 0; k < kTile / 16; k++)
                    mma(tb + dcol, mnmajor(g, kTile, k), mnmajor(h, kTile, k), kIdDW, (!first || k > 0));
#pragma unroll
                for (uint32_t k = 0; k < kHidden / 16; k++)
                    mma(tb + kColDH, kmajor(g, kTile, k), mnmajor(w, kHidden, k), kIdDH, k > 0);
                commit(&bar);
            }
            wait_mma();
            epilogue_mask(lane + kColDH, Hs + (l - 1) * kHBytes, G + (cur ^ 1u) * kHBytes, t);
            sync_for_mma();
            if (abort_s) { aborted = true; break; }
            cur ^= 1u;
        }
        if (aborted) break;
        // dW0 += g0^T X
        if (t == 0) {
            const uint32_t g = sG + cur * kHBytes;
#pragma unroll
            for (uint32_t k = 0; k < kTile / 16; k++)
                mma(tb + kColDW0, mnmajor(g, kTile, k), mnmajor(sX, kTile, k), kIdDW0, (!first || k > 0));
            commit(&bar);
        }
        wait_mma();
        sync_for_mma();
        if (abort_s) { aborted = true; break; }
        first = false;
    }

    if (aborted) {
        if (t == 0) { atomicOr(error_flags, kErrTimeout); mbar_wait(&bar, phase); }
        fence_before_sync();
        __syncthreads();
    } else if (!first) {
        // M=64 accumulators: warp w holds rows 16w..16w+15 in lanes 0..15.
        float *out = partials + (size_t)blockIdx.x * kParams;
        const uint32_t row = warp * 16u + (t & 31u);
        const bool has_row = (t & 31u) < 16u;
        float v[32];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            tmem_ld32(lane + kColDW0 + 32u * c, v);
            if (has_row)
                for (int j = 0; j < 32; j++) out[row * kInputs + 32 * c + j] = v[j];
        }
        for (int l = 0; l < 3; l++) {
#pragma unroll
            for (int c = 0; c < 2; c++) {
                tmem_ld32(lane + kColDW1 + 64u * l + 32u * c, v);
                if (has_row)
                    for (int j = 0; j < 32; j++) out[kParamsW0 + l * kParamsW + row * kHidden + 32 * c + j] = v[j];
            }
        }
        float v16[16];
        tmem_ld16w(lane + kColDW4, v16);      // dW4^T: row = input unit, column = output
        if (has_row)
            for (int o = 0; o < kOutputs; o++) out[kParamsW0 + 3 * kParamsW + o * kHidden + row] = v16[o];
        fence_before_sync();
    } else {
        // no tile: an all-zero partial row keeps the reduction uniform
        float *out = partials + (size_t)blockIdx.x * kParams;
        for (uint32_t p = t; p < (uint32_t)kParams; p += blockDim.x) out[p] = 0.0f;
    }
    for (int o = 16; o; o >>= 1) loss += __shfl_down_sync(0xFFFFFFFFu, loss, o);
    if ((t & 31u) == 0) loss_s[warp] = loss;
    __syncthreads();
    if (t == 0) loss_partials[blockIdx.x] = (loss_s[0] + loss_s[1]) + (loss_s[2] + loss_s[3]);
    if (warp == 0) tmem_free(tb, 512);
}

// Image offset of parameter p.
SLIM_N uint32_t param_offset(uint32_t p) {
    if (p < (uint32_t)kParamsW0) return img_off(kHidden, p / kInputs, p % kInputs);
    p -= kParamsW0;
    if (p < 3u * kParamsW) return kImgOff1 + (p / kParamsW) * kImgW + img_off(kHidden, (p % kParamsW) / kHidden, p % kHidden);
    p -= 3u * kParamsW;
    return kImgOff4 + img_off(kOutPad, p / kHidden, p % kHidden);
}

__global__ void k_nrc_adam(float *__restrict__ params, float *__restrict__ m, float *__restrict__ v,
                           const float *__restrict__ partials, const float *__restrict__ loss_partials,
                           float *__restrict__ grad, float *__restrict__ loss, uint8_t *__restrict__ image, AdamArgs a,
                           uint32_t n_max, const uint32_t *count, uint32_t offset) {
    uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t n = step_samples(n_max, count, offset);
    if (!n) return;                                  // empty step: no update
    const float scale = 1.0f / (3.0f * (float)n);
    const float t = (float)*a.step;
    const float bias1 = 1.0f / (1.0f - powf(a.beta1, t)), bias2 = 1.0f / (1.0f - powf(a.beta2, t));
    if (p == 0) {
        float s = 0.0f;
        for (uint32_t b = 0; b < a.parts; b++) s += loss_partials[b];
        *loss = s * scale;
    }
    if (p >= (uint32_t)kParams) return;
    float g = 0.0f;
    for (uint32_t b = 0; b < a.parts; b++) g += partials[(size_t)b * kParams + p];
    g *= scale;
    grad[p] = g;
    float mm = a.beta1 * m[p] + (1.0f - a.beta1) * g;
    float vv = a.beta2 * v[p] + (1.0f - a.beta2) * g * g;
    m[p] = mm;
    v[p] = vv;
    float w = params[p] - a.lr * (mm * bias1) / (sqrtf(vv * bias2) + a.eps);
    params[p] = w;
    *(unsigned short *)(image + param_offset(p)) = (unsigned short)bf16_bits(w);
}

__global__ void k_nrc_pack(const float *__restrict__ params, uint8_t *__restrict__ image) {
    uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < (uint32_t)kParams) *(unsigned short *)(image + param_offset(p)) = (unsigned short)bf16_bits(params[p]);
}

#undef SLIM_N

// ---- launchers ------------------------------------------------------------------
namespace {
int sm_count() {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}
}  // namespace

// CTAs of a training step: one per 128-sample tile, at most one per SM and at
// most SLIM_NRC_TRAIN_MAX_CTAS (0: no cap); a CTA loops over several tiles.
// A training CTA holds 166 KB of shared memory, which on its SM is taken from
// the L1 cache that the traversal kernels running beside an overlapped
// training step read their nodes through: config 4 (65,536 samples per
// frame) 1.694 ms per cache frame with 128 CTAs per step, 1.648 with 64,
// 1.636 with 32.
#ifndef SLIM_NRC_TRAIN_MAX_CTAS
#define SLIM_NRC_TRAIN_MAX_CTAS 32
#endif
int train_grid(uint32_t samples) {
    uint32_t tiles = (samples + kTile - 1) / kTile;
    uint32_t g = (uint32_t)sm_count();
    if (SLIM_NRC_TRAIN_MAX_CTAS > 0 && g > (uint32_t)SLIM_NRC_TRAIN_MAX_CTAS) g = SLIM_NRC_TRAIN_MAX_CTAS;
    return (int)(tiles < g ? (tiles ? tiles : 1) : g);
}

cudaError_t prepare() {
    cudaError_t e = cudaFuncSetAttribute(k_nrc_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, kInferSmem);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_nrc_train, cudaFuncAttributeMaxDynamicSharedMemorySize, kTrainSmem);
}

cudaError_t launch_infer(const float4 *features, const uint32_t *count, uint32_t n, uint32_t capacity, float4 *radiance,
                         const uint8_t *weight_image, uint32_t *error_flags, cudaStream_t stream) {
    uint32_t bound = count ? capacity : n;
    uint32_t tiles = (bound + kTile - 1) / kTile;
    if (!tiles) return cudaSuccess;
    uint32_t g = 2u * (uint32_t)sm_count();
    if (tiles < g) g = tiles;
    k_nrc_infer<<<g, 128, kInferSmem, stream>>>(features, count, n, radiance, weight_image, error_flags);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_train_step(const float4 *features, const float4 *targets, uint32_t samples, const uint32_t *count,
                              uint32_t offset, float *params, float *adam_m, float *adam_v, uint8_t *weight_image,
                              float *partials, float *loss_partials, float *grad, float *loss, const AdamArgs &adam,
                              uint32_t *error_flags, cudaStream_t stream) {
    if (!samples) return cudaSuccess;
    int g = train_grid(samples);
    k_nrc_train<<<g, 128, kTrainSmem, stream>>>(features, targets, samples, count, offset, weight_image, partials,
                                                 loss_partials, adam.step, error_flags);
    count_launch();
    AdamArgs a = adam;
    a.parts = (uint32_t)g;
    k_nrc_adam<<<(kParams + 255) / 256, 256, 0, stream>>>(params, adam_m, adam_v, partials, loss_partials, grad, loss,
                                                          weight_image, a, samples, count, offset);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_pack_weights(const float *params, uint8_t *weight_image, cudaStream_t stream) {
    cudaError_t e = cudaMemsetAsync(weight_image, 0, kImgBytes, stream);
    if (e != cudaSuccess) return e;
    k_nrc_pack<<<(kParams + 255) / 256, 256, 0, stream>>>(params, weight_image);
    count_launch();
    return cudaGetLastError();
}

}  // namespace nrc
}  // namespace slim
