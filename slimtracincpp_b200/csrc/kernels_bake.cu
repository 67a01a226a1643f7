// Texel-quad texture baker on the device: bmp2texture's conversion
// (bmp2texture.cpp:24-335), the same bytes as the host restatement in
// texture_baker.cpp for every image and flag set.
//
//   k_bake_texels  8-bit components -> float texels (the gamma curve comes
//                  from a 256-entry table the host fills with its own powf,
//                  so both bakers see the same values); normal maps decoded
//                  (bmp2texture.cpp:306-321); cube strips split into faces
//   k_bake_quads   one thread per texel quad.  The reference fills quads by
//                  walking texels in row order, each texel writing the quad
//                  corners around it plus border and wrap corners, later
//                  writes replacing earlier ones (TextureMipLoader::load,
//                  bmp2texture.cpp:36-131).  Only texels of the rows and
//                  columns beside a quad, and the opposite border under
//                  wrap, write to it, so the thread replays those (at most
//                  nine) texels' writes in row order and keeps the last
//   k_bake_mip     the next mip's texels: the 2x2 box filter of the larger
//                  mip's inner quads (loadMips, bmp2texture.cpp:212-237),
//                  whose corners are always the four texels themselves
//   k_cube_seams   one thread: the cube faces' seam writes and corner
//                  blends (bmp2texture.cpp:133-209), in the reference's
//                  order, after the fill
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <vector>

#include "host_common.h"
#include "kernels.h"

namespace slim {
namespace {

constexpr float kByteScale = 0.00392156862f;   // componentsToPixel's 1/255

struct BakeLevel {
    uint32_t width, height;
    size_t texel_offset;   // into the texel buffer (float4), one zero texel of slack after each level
    size_t quad_offset;    // into the quad output
};

__device__ inline uint8_t to_byte(float v) { return (uint8_t)(v * 255.0f); }

// Pixel::lerpTo (core/base.h:1100-1105)
__device__ inline float4 lerp_px(float4 from, float4 to, float by) {
    float4 o;
    o.x = fmaf(to.x - from.x, by, from.x);
    o.y = fmaf(to.y - from.y, by, from.y);
    o.z = fmaf(to.z - from.z, by, from.z);
    o.w = from.w + (to.w - from.w) * by;
    return o;
}

// texels: (r, g, b, a).  Image pixel (x, y) of a cube's 6h x h strip goes
// to the 4h-wide main strip, the top face or the bottom face.
__global__ void k_bake_texels(const uint8_t *__restrict__ bgr, uint32_t width, uint32_t height, uint32_t channels,
                              const float *__restrict__ table, bool normal, bool cube, float4 *main,
                              float4 *top, float4 *bottom) {
    const size_t n = (size_t)width * height;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const uint8_t *c = bgr + i * channels;
        float4 p;
        p.z = table[c[0]];
        p.y = table[c[1]];
        p.x = table[c[2]];
        p.w = channels == 4 ? (float)c[3] * kByteScale : 0.0f;
        if (normal) {
            float r = p.x * 2.0f - 1.0f;
            float g = p.y * 2.0f - 1.0f;
            float l_rcp = 1.0f / sqrtf(r * r + g * g + 1.0f);
            r *= l_rcp;
            g *= l_rcp;
            float b = sqrtf(1.0f - r * r - g * g);
            p.x = r * 0.5f + 0.5f;
            p.y = g * 0.5f + 0.5f;
            p.z = b * 0.5f + 0.5f;
        }
        if (!cube) {
            main[i] = p;
            continue;
        }
        const uint32_t y = (uint32_t)(i / width), x = (uint32_t)(i % width), face = height, strip = 4 * face;
        if (x < strip) main[(size_t)strip * y + x] = p;
        else if (x < strip + face) top[(size_t)face * y + (x - strip)] = p;
        else bottom[(size_t)face * y + (x - strip - face)] = p;
    }
}

// Corner slots of a quad: 0 TL, 1 TR, 2 BL, 3 BR.
struct QuadTarget {
    uint32_t qx, qy;
    float4 c[4];
    __device__ void put(uint32_t x, uint32_t y, int corner, float4 v) {
        if (x == qx && y == qy) c[corner] = v;
    }
};

// The writes of texel (x, y) of a w x h mip, in the reference's order.
__device__ void replay_texel(QuadTarget &q, uint32_t x, uint32_t y, uint32_t w, uint32_t h, bool wrap, float4 v) {
    const bool L = x == 0, R = x == w - 1, T = y == 0, B = y == h - 1;
    q.put(x, y, 3, v);
    q.put(x + 1, y, 2, v);
    q.put(x, y + 1, 1, v);
    q.put(x + 1, y + 1, 0, v);
    if (L) {
        q.put(x, y, 2, v);
        q.put(x, y + 1, 0, v);
    } else if (R) {
        q.put(x + 1, y, 3, v);
        q.put(x + 1, y + 1, 1, v);
    }
    if (wrap) {
        if (L) {
            q.put(w, y, 3, v);
            q.put(w, y + 1, 1, v);
        } else if (R) {
            q.put(0, y, 2, v);
            q.put(0, y + 1, 0, v);
        }
        if (T) {
            q.put(x, h, 3, v);
            q.put(x + 1, h, 2, v);
            if (L) q.put(w, h, 3, v);
            else if (R) q.put(0, h, 2, v);
        } else if (B) {
            q.put(x, 0, 1, v);
            q.put(x + 1, 0, 0, v);
            if (L) q.put(w, 0, 1, v);
            else if (R) q.put(0, 0, 0, v);
        }
    } else {
        if (T) {
            q.put(x, y, 1, v);
            q.put(x + 1, y, 0, v);
            if (L) q.put(x, y, 0, v);
            else if (R) q.put(x + 1, y, 1, v);
        } else if (B) {
            q.put(x, y + 1, 3, v);
            q.put(x + 1, y + 1, 2, v);
            if (L) q.put(x, y + 1, 2, v);
            else if (R) q.put(x + 1, y + 1, 3, v);
        }
    }
}

__device__ inline void store_quad(SlimTexelQuad *out, const float4 c[4]) {
    SlimTexelQuad o;
    for (int k = 0; k < 4; k++) {
        o.R[k] = to_byte(c[k].x);
        o.G[k] = to_byte(c[k].y);
        o.B[k] = to_byte(c[k].z);
    }
    *out = o;
}

__global__ void k_bake_quads(const float4 *__restrict__ texels, uint32_t w, uint32_t h, bool wrap,
                             SlimTexelQuad *out) {
    const uint32_t stride = w + 1;
    const size_t n = (size_t)stride * (h + 1);
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        QuadTarget q;
        q.qx = (uint32_t)(i % stride);
        q.qy = (uint32_t)(i / stride);
        for (int k = 0; k < 4; k++) q.c[k] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        // texel rows and columns that write this quad, ascending
        uint32_t rows[3], cols[3], nr = 0, nc = 0;
        if (wrap && q.qy == h && h > 1) rows[nr++] = 0;            // top row wraps to the bottom line
        if (q.qy >= 1) rows[nr++] = q.qy - 1;
        if (q.qy < h && !(nr && rows[nr - 1] == q.qy)) rows[nr++] = q.qy;
        if (wrap && q.qy == 0 && h - 1 > q.qy && !(nr && rows[nr - 1] == h - 1)) rows[nr++] = h - 1;
        if (wrap && q.qx == w && w > 1) cols[nc++] = 0;
        if (q.qx >= 1) cols[nc++] = q.qx - 1;
        if (q.qx < w && !(nc && cols[nc - 1] == q.qx)) cols[nc++] = q.qx;
        if (wrap && q.qx == 0 && w - 1 > q.qx && !(nc && cols[nc - 1] == w - 1)) cols[nc++] = w - 1;
        for (uint32_t a = 0; a < nr; a++)
            for (uint32_t b = 0; b < nc; b++)
                replay_texel(q, cols[b], rows[a], w, h, wrap, texels[(size_t)w * rows[a] + cols[b]]);
        store_quad(out + i, q.c);
    }
}

__global__ void k_bake_mip(const float4 *__restrict__ prev, uint32_t prev_w, float4 *next, uint32_t w, uint32_t h) {
    const size_t n = (size_t)w * h;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const uint32_t x = (uint32_t)(i % w), y = (uint32_t)(i / w);
        const float4 *r0 = prev + (size_t)prev_w * (2 * y) + 2 * x, *r1 = r0 + prev_w;
        const float4 tl = r0[0], tr = r0[1], bl = r1[0], br = r1[1];
        float4 t;
        t.x = 0.25f * (tl.x + tr.x + bl.x + br.x);
        t.y = 0.25f * (tl.y + tr.y + bl.y + br.y);
        t.z = 0.25f * (tl.z + tr.z + bl.z + br.z);
        t.w = 0.0f;
        next[i] = t;
    }
}

// A corner write of the seam pass: bytes of `v` into corner `k` of quad
// `i` of a level of `count` quads.  The reference's main-strip pass writes
// two quads past the strip's last row, into its loader's slack: dropped.
__device__ inline void seam_put(SlimTexelQuad *quads, size_t count, size_t i, int k, float4 v) {
    if (i >= count) return;
    quads[i].R[k] = to_byte(v.x);
    quads[i].G[k] = to_byte(v.y);
    quads[i].B[k] = to_byte(v.z);
}

__global__ void k_cube_seams(const float4 *main, const float4 *top_face, const float4 *bottom_face, uint32_t face,
                             SlimTexelQuad *main_quads, SlimTexelQuad *top_quads, SlimTexelQuad *bottom_quads) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const uint32_t h = face, w = h, s = w * h, last = w - 1, last_row = w * last, last_texel = s - 1;
    const uint32_t Lo0 = 0, Fo0 = w, Ro0 = w * 2, Bo0 = w * 3;
    // main strip (4w x h texels, 4w + 1 quads a row)
    {
        const uint32_t width = 4 * w, stride = width + 1;
        const size_t count = (size_t)stride * (h + 1), bottom = (size_t)h * stride;
        const uint32_t quad_w = (w + 1) * 4;
        uint32_t Lo = Lo0, Fo = Fo0, Ro = Ro0, Bo = Bo0;
        for (uint32_t i = 0; i < h; i++, Lo++, Ro++, Fo++, Bo++) {
            float4 v = top_face[w * i];
            seam_put(main_quads, count, 1 + Lo, 0, v); seam_put(main_quads, count, Lo, 1, v);
            v = top_face[last_row + i];
            seam_put(main_quads, count, 1 + Fo, 0, v); seam_put(main_quads, count, Fo, 1, v);
            v = top_face[last_texel - (w * i)];
            seam_put(main_quads, count, 1 + Ro, 0, v); seam_put(main_quads, count, Ro, 1, v);
            v = top_face[w - i];
            seam_put(main_quads, count, 1 + Bo, 0, v); seam_put(main_quads, count, Bo, 1, v);
            v = bottom_face[w * (last - i)];
            seam_put(main_quads, count, bottom + 1 + Lo, 2, v); seam_put(main_quads, count, bottom + Lo, 3, v);
            v = bottom_face[i];
            seam_put(main_quads, count, bottom + 1 + Fo, 2, v); seam_put(main_quads, count, bottom + Fo, 3, v);
            v = bottom_face[w * i + last];
            seam_put(main_quads, count, bottom + 1 + Ro, 2, v); seam_put(main_quads, count, bottom + Ro, 3, v);
            v = bottom_face[last_row + (w - i)];
            seam_put(main_quads, count, bottom + 1 + Bo, 2, v); seam_put(main_quads, count, bottom + Bo, 3, v);
        }
        seam_put(main_quads, count, 0, 0, lerp_px(top_face[0], main[width - 1], 0.5f));
        seam_put(main_quads, count, quad_w - 1, 1, lerp_px(top_face[0], main[0], 0.5f));
        seam_put(main_quads, count, bottom, 2, lerp_px(bottom_face[last_row], main[(size_t)width * last], 0.5f));
        seam_put(main_quads, count, bottom + quad_w - 1, 3, lerp_px(bottom_face[last_row], main[0], 0.5f));
    }
    const uint32_t stride = w + 1;
    const size_t count = (size_t)stride * (h + 1), bottom = (size_t)h * stride;
    // top face
    {
        const float4 *lf = main + Lo0, *ff = main + Fo0, *rf = main + Ro0, *bf = main + Bo0;
        seam_put(top_quads, count, 0, 0, lerp_px(lf[0], bf[last], 0.5f));
        seam_put(top_quads, count, w, 1, lerp_px(bf[0], rf[last], 0.5f));
        seam_put(top_quads, count, bottom, 2, lerp_px(ff[0], lf[last], 0.5f));
        seam_put(top_quads, count, bottom + w, 3, lerp_px(rf[0], ff[last], 0.5f));
        rf += last;
        bf += last;
        size_t lc = 0, rc = w;
        for (uint32_t i = 0; i < h; i++, lc += stride, rc += stride, lf++, ff++, rf--, bf--) {
            seam_put(top_quads, count, 1 + i, 0, *bf); seam_put(top_quads, count, i, 1, *bf);
            seam_put(top_quads, count, bottom + 1 + i, 2, *ff); seam_put(top_quads, count, bottom + i, 3, *ff);
            seam_put(top_quads, count, lc, 2, *lf); seam_put(top_quads, count, lc + stride, 0, *lf);
            seam_put(top_quads, count, rc, 3, *rf); seam_put(top_quads, count, rc + stride, 1, *rf);
        }
    }
    // bottom face
    {
        const uint32_t mlast = w * 4 * last;
        const float4 *lf = main + Lo0 + mlast, *ff = main + Fo0 + mlast, *rf = main + Ro0 + mlast,
                     *bf = main + Bo0 + mlast;
        seam_put(bottom_quads, count, 0, 0, lerp_px(ff[0], lf[last], 0.5f));
        seam_put(bottom_quads, count, w, 1, lerp_px(rf[0], ff[last], 0.5f));
        seam_put(bottom_quads, count, bottom, 2, lerp_px(lf[0], bf[last], 0.5f));
        seam_put(bottom_quads, count, bottom + w, 3, lerp_px(bf[0], rf[last], 0.5f));
        lf += last;
        bf += last;
        size_t lc = 0, rc = w;
        for (uint32_t i = 0; i < h; i++, lc += stride, rc += stride, lf--, ff++, rf++, bf--) {
            seam_put(bottom_quads, count, 1 + i, 0, *ff); seam_put(bottom_quads, count, i, 1, *ff);
            seam_put(bottom_quads, count, bottom + 1 + i, 2, *bf); seam_put(bottom_quads, count, bottom + i, 3, *bf);
            seam_put(bottom_quads, count, lc, 2, *lf); seam_put(bottom_quads, count, lc + stride, 0, *lf);
            seam_put(bottom_quads, count, rc, 3, *rf); seam_put(bottom_quads, count, rc + stride, 1, *rf);
        }
    }
}

uint32_t grid_for(size_t n) {
    size_t g = (n + 255) / 256;
    return (uint32_t)(g < 148 * 16 ? (g ? g : 1) : 148 * 16);
}

struct DeviceBlock {
    void *p = nullptr;
    ~DeviceBlock() { if (p) cudaFree(p); }
};

}  // namespace

int bake_texture_gpu(const uint8_t *bgr, uint32_t width, uint32_t height, uint32_t channels, uint32_t flags,
                     SlimTexture *texture, SlimTextureMip *mips, SlimTexelQuad *quads, uint32_t *mip_count,
                     uint32_t *quad_count, cudaStream_t stream) {
    if (!bgr || !texture || !mip_count || !quad_count || !width || !height || (channels != 3 && channels != 4))
        return set_error(SLIM_ERR_ARGUMENT, "slimBakeTextureOnGPU: bad arguments");
    const bool cube = (flags & SLIM_IMAGE_CUBEMAP) != 0;
    if (cube && width != 6 * height) return set_error(SLIM_ERR_ARGUMENT, "slimBakeTextureOnGPU: a cube map is 6h x h");
    if ((uint64_t)width * height > (1ull << 28)) return set_error(SLIM_ERR_LIMIT, "slimBakeTextureOnGPU: image too large");
    uint32_t f = flags & (SLIM_IMAGE_LINEAR | SLIM_IMAGE_MIPMAP | SLIM_IMAGE_WRAP | SLIM_IMAGE_NORMAL | SLIM_IMAGE_CUBEMAP);
    if (channels == 4) f |= SLIM_IMAGE_ALPHA;
    if (cube) f &= ~(SLIM_IMAGE_WRAP | SLIM_IMAGE_NORMAL | SLIM_IMAGE_MIPMAP);
    const bool linear = (f & SLIM_IMAGE_LINEAR) != 0, wrap = (f & SLIM_IMAGE_WRAP) != 0;
    std::vector<BakeLevel> levels;
    if (cube) {
        levels.push_back({4 * height, height, 0, 0});
        levels.push_back({height, height, 0, 0});
        levels.push_back({height, height, 0, 0});
    } else {
        levels.push_back({width, height, 0, 0});
        if (f & SLIM_IMAGE_MIPMAP)
            for (uint32_t w = width, h = height; w > 4 && h > 4;) {
                w /= 2;
                h /= 2;
                levels.push_back({w, h, 0, 0});
            }
    }
    size_t texel_total = 0, quad_total = 0;
    for (BakeLevel &l : levels) {
        l.texel_offset = texel_total;
        l.quad_offset = quad_total;
        texel_total += (size_t)l.width * l.height + 1;   // a zero texel of slack: the seam pass reads one past a face
        quad_total += (size_t)(l.width + 1) * (l.height + 1);
    }
    if (quad_total > 0xFFFFFFFFull) return set_error(SLIM_ERR_LIMIT, "slimBakeTextureOnGPU: too many texel quads");
    memset(texture, 0, sizeof(*texture));
    texture->width = width;
    texture->height = height;
    texture->size = width * height;
    texture->stride = width;
    texture->mip_count = (uint32_t)levels.size();
    texture->flags = f;
    *mip_count = (uint32_t)levels.size();
    *quad_count = (uint32_t)quad_total;
    if (!quads || !mips) return SLIM_OK;   // sizing call

    float table[256];
    for (int c = 0; c < 256; c++) table[c] = bake_component((uint8_t)c, linear);
    const size_t image_bytes = (size_t)width * height * channels;
    const size_t texel_bytes = texel_total * sizeof(float4), quad_bytes = quad_total * sizeof(SlimTexelQuad);
    const size_t off_texels = 0, off_quads = texel_bytes, off_table = off_quads + ((quad_bytes + 255) & ~(size_t)255),
                 off_image = off_table + 256 * sizeof(float);
    DeviceBlock block;
    cudaError_t e = cudaMalloc(&block.p, off_image + image_bytes);
    if (e != cudaSuccess) return set_error(SLIM_ERR_CUDA, "slimBakeTextureOnGPU: device memory");
    char *base = static_cast<char *>(block.p);
    float4 *texels = reinterpret_cast<float4 *>(base + off_texels);
    SlimTexelQuad *d_quads = reinterpret_cast<SlimTexelQuad *>(base + off_quads);
    float *d_table = reinterpret_cast<float *>(base + off_table);
    uint8_t *d_image = reinterpret_cast<uint8_t *>(base + off_image);
#define BAKE_CUDA(x)                                                                    \
    do {                                                                                \
        if ((e = (x)) != cudaSuccess) return set_error(SLIM_ERR_CUDA, cudaGetErrorString(e)); \
    } while (0)
    BAKE_CUDA(cudaMemsetAsync(texels, 0, texel_bytes, stream));
    BAKE_CUDA(cudaMemcpyAsync(d_table, table, sizeof(table), cudaMemcpyHostToDevice, stream));
    BAKE_CUDA(cudaMemcpyAsync(d_image, bgr, image_bytes, cudaMemcpyHostToDevice, stream));
    float4 *t0 = texels + levels[0].texel_offset;
    float4 *t1 = cube ? texels + levels[1].texel_offset : nullptr, *t2 = cube ? texels + levels[2].texel_offset : nullptr;
    k_bake_texels<<<grid_for((size_t)width * height), 256, 0, stream>>>(
        d_image, width, height, channels, d_table, !cube && (f & SLIM_IMAGE_NORMAL), cube, t0, t1, t2);
    count_launch();
    for (size_t m = 0; m < levels.size(); m++) {
        const BakeLevel &l = levels[m];
        if (!cube && m > 0) {
            const BakeLevel &p = levels[m - 1];
            k_bake_mip<<<grid_for((size_t)l.width * l.height), 256, 0, stream>>>(
                texels + p.texel_offset, p.width, texels + l.texel_offset, l.width, l.height);
            count_launch();
        }
        k_bake_quads<<<grid_for((size_t)(l.width + 1) * (l.height + 1)), 256, 0, stream>>>(
            texels + l.texel_offset, l.width, l.height, wrap, d_quads + l.quad_offset);
        count_launch();
    }
    if (cube) {
        k_cube_seams<<<1, 1, 0, stream>>>(t0, t1, t2, height, d_quads + levels[0].quad_offset,
                                          d_quads + levels[1].quad_offset, d_quads + levels[2].quad_offset);
        count_launch();
    }
    BAKE_CUDA(cudaGetLastError());
    BAKE_CUDA(cudaMemcpyAsync(quads, d_quads, quad_bytes, cudaMemcpyDeviceToHost, stream));
    BAKE_CUDA(cudaStreamSynchronize(stream));
#undef BAKE_CUDA
    for (size_t m = 0; m < levels.size(); m++) {
        mips[m].width = levels[m].width;
        mips[m].height = levels[m].height;
        mips[m].texel_quads = quads + levels[m].quad_offset;
    }
    texture->mips = mips;
    return SLIM_OK;
}

}  // namespace slim
