// Texel-quad texture baker: the reference's bmp2texture conversion
// (bmp2texture.cpp:24-335) from the 8-bit components its loadBitmap returns
// (platforms/win32_bitmap.h:122-160: B, G, R[, A] per pixel, rows after the
// loader's flip).  Each texel is replicated into the four quads that share
// it, so a bilinear tap reads one 12-byte TexelQuad; borders are clamped or
// wrapped, cube-map strips get their seams from the neighbouring faces, and
// smaller mips are 2x2 box-filtered from the larger one's quads.  The quad
// fill order and the float arithmetic follow the reference step by step:
// the output is compared byte for byte with its .texture files.
#include <cmath>
#include <cstring>
#include <vector>

#include "host_common.h"

namespace slim {
namespace {

struct Px { float r = 0, g = 0, b = 0, a = 0; };
struct PxQuad { Px TL, TR, BL, BR; };

// Pixel::lerpTo (core/base.h:1100-1105)
Px lerp(const Px &from, const Px &to, float by) {
    Px o;
    o.r = fmaf(to.r - from.r, by, from.r);
    o.g = fmaf(to.g - from.g, by, from.g);
    o.b = fmaf(to.b - from.b, by, from.b);
    o.a = from.a + (to.a - from.a) * by;
    return o;
}

enum CubeMode { CubeNone = 0, CubeMain, CubeTop, CubeBottom };

struct MipLoader {
    uint32_t width = 0, height = 0;
    std::vector<Px> texels;
    std::vector<PxQuad> quads;

    // The cube-map seam fill reads one texel past a face
    // (bmp2texture.cpp:140, i == 0) and writes two quads past the strip
    // (bmp2texture.cpp:145, quad_w is 4(w+1) for a 4w+1-quad row); the
    // slack keeps both inside these buffers and outside the baked output.
    static constexpr size_t kTexelSlack = 1, kQuadSlack = 4;
    size_t quad_count() const { return (size_t)(width + 1) * (height + 1); }

    void init(uint32_t w, uint32_t h) {
        width = w;
        height = h;
        texels.assign((size_t)w * h + kTexelSlack, Px{});
        quads.assign(quad_count() + kQuadSlack, PxQuad{});
    }

    // TextureMipLoader::load (bmp2texture.cpp:36-209)
    void load(bool wrap, CubeMode mode = CubeNone, const Px *main_faces = nullptr, const Px *top_face = nullptr,
              const Px *bottom_face = nullptr) {
        const uint32_t stride = width + 1, last_x = width - 1, last_y = height - 1, l = 0, r = width;
        const Px *texel = texels.data();
        PxQuad *top_line = quads.data();
        PxQuad *bottom_line = top_line + (size_t)height * stride;
        PxQuad *cur = top_line, *next = top_line + stride;
        for (uint32_t y = 0; y < height; y++, cur += stride, next += stride) {
            bool T = y == 0, B = y == last_y;
            for (uint32_t x = 0; x < width; x++, texel++) {
                PxQuad *TL = cur + x, *TR = cur + x + 1, *BL = next + x, *BR = next + x + 1;
                bool L = x == 0, R = x == last_x;
                TL->BR = TR->BL = BL->TR = BR->TL = *texel;
                if (L) TL->BL = BL->TL = *texel;
                else if (R) TR->BR = BR->TR = *texel;
                if (wrap) {
                    if (L) cur[r].BR = next[r].TR = *texel;
                    else if (R) cur[l].BL = next[l].TL = *texel;
                    if (T) {
                        bottom_line[x].BR = bottom_line[x + 1].BL = *texel;
                        if (L) bottom_line[r].BR = *texel;
                        else if (R) bottom_line[l].BL = *texel;
                    } else if (B) {
                        top_line[x].TR = top_line[x + 1].TL = *texel;
                        if (L) top_line[r].TR = *texel;
                        else if (R) top_line[l].TL = *texel;
                    }
                } else {
                    if (T) {
                        TL->TR = TR->TL = *texel;
                        if (L) TL->TL = *texel;
                        else if (R) TR->TR = *texel;
                    } else if (B) {
                        BL->BR = BR->BL = *texel;
                        if (L) BL->BL = *texel;
                        else if (R) BR->BR = *texel;
                    }
                }
            }
        }
        if (mode == CubeNone) return;
        const uint32_t h = height, w = h, s = w * h, last = w - 1, last_row = w * last, last_texel = s - 1;
        uint32_t quad_w = (w + 1) * 4;
        uint32_t Lo = 0, Fo = w, Ro = w * 2, Bo = w * 3;
        switch (mode) {
            case CubeMain:
                for (uint32_t i = 0; i < h; i++, Lo++, Ro++, Fo++, Bo++) {
                    top_line[1 + Lo].TL = top_line[Lo].TR = top_face[w * i];
                    top_line[1 + Fo].TL = top_line[Fo].TR = top_face[last_row + i];
                    top_line[1 + Ro].TL = top_line[Ro].TR = top_face[last_texel - (w * i)];
                    top_line[1 + Bo].TL = top_line[Bo].TR = top_face[w - i];
                    bottom_line[1 + Lo].BL = bottom_line[Lo].BR = bottom_face[w * (last - i)];
                    bottom_line[1 + Fo].BL = bottom_line[Fo].BR = bottom_face[i];
                    bottom_line[1 + Ro].BL = bottom_line[Ro].BR = bottom_face[w * i + last];
                    bottom_line[1 + Bo].BL = bottom_line[Bo].BR = bottom_face[last_row + (w - i)];
                }
                top_line[0].TL = lerp(top_face[0], texels[width - 1], 0.5f);
                top_line[quad_w - 1].TR = lerp(top_face[0], texels[0], 0.5f);
                bottom_line[0].BL = lerp(bottom_face[last_row], texels[width * last], 0.5f);
                bottom_line[quad_w - 1].BR = lerp(bottom_face[last_row], texels[0], 0.5f);
                break;
            case CubeTop: {
                const Px *lf = main_faces + Lo, *ff = main_faces + Fo, *rf = main_faces + Ro, *bf = main_faces + Bo;
                top_line[0].TL = lerp(lf[0], bf[last], 0.5f);
                top_line[w].TR = lerp(bf[0], rf[last], 0.5f);
                bottom_line[0].BL = lerp(ff[0], lf[last], 0.5f);
                bottom_line[w].BR = lerp(rf[0], ff[last], 0.5f);
                rf += last;
                bf += last;
                PxQuad *lc = quads.data(), *rc = quads.data() + w;
                quad_w = w + 1;
                for (uint32_t i = 0; i < h; i++, lc += quad_w, rc += quad_w, lf++, ff++, rf--, bf--) {
                    top_line[1 + i].TL = top_line[i].TR = *bf;
                    bottom_line[1 + i].BL = bottom_line[i].BR = *ff;
                    lc[0].BL = lc[quad_w].TL = *lf;
                    rc[0].BR = rc[quad_w].TR = *rf;
                }
            } break;
            case CubeBottom: {
                uint32_t mstride = w * 4, mlast = mstride * last;
                Lo += mlast; Ro += mlast; Fo += mlast; Bo += mlast;
                const Px *lf = main_faces + Lo, *ff = main_faces + Fo, *rf = main_faces + Ro, *bf = main_faces + Bo;
                top_line[0].TL = lerp(ff[0], lf[last], 0.5f);
                top_line[w].TR = lerp(rf[0], ff[last], 0.5f);
                bottom_line[0].BL = lerp(lf[0], bf[last], 0.5f);
                bottom_line[w].BR = lerp(bf[0], rf[last], 0.5f);
                lf += last;
                bf += last;
                PxQuad *lc = quads.data(), *rc = quads.data() + w;
                quad_w = w + 1;
                for (uint32_t i = 0; i < h; i++, lc += quad_w, rc += quad_w, lf--, ff++, rf++, bf--) {
                    top_line[1 + i].TL = top_line[i].TR = *ff;
                    bottom_line[1 + i].BL = bottom_line[i].BR = *bf;
                    lc[0].BL = lc[quad_w].TL = *lf;
                    rc[0].BR = rc[quad_w].TR = *rf;
                }
            } break;
            default: break;
        }
    }
};

// componentsToPixel with gamma 2.2 (platforms/win32_bitmap.h:12-33)
Px component_pixel(const uint8_t *c, uint32_t channels, bool linear) {
    const float k = 0.00392156862f;
    Px p;
    p.b = (float)c[0] * k;
    p.g = (float)c[1] * k;
    p.r = (float)c[2] * k;
    p.a = channels == 4 ? (float)c[3] * k : 0.0f;
    if (!linear) {
        p.r = powf(p.r, 2.2f);
        p.g = powf(p.g, 2.2f);
        p.b = powf(p.b, 2.2f);
    }
    return p;
}

inline uint8_t to_byte(float v) { return (uint8_t)(v * 255.0f); }

}  // namespace

// The colour value component_pixel gives an 8-bit component: the device
// baker's lookup table.
float bake_component(uint8_t c, bool linear) {
    const uint8_t bgr[3] = {c, c, c};
    return component_pixel(bgr, 3, linear).r;
}

int bake_texture(const uint8_t *bgr, uint32_t width, uint32_t height, uint32_t channels, uint32_t flags,
                 SlimTexture *texture, SlimTextureMip *mips, SlimTexelQuad *quads, uint32_t *mip_count,
                 uint32_t *quad_count) {
    if (!bgr || !texture || !mip_count || !quad_count || !width || !height || (channels != 3 && channels != 4))
        return set_error(SLIM_ERR_ARGUMENT, "slimBakeTexture: bad arguments");
    bool cube = (flags & SLIM_IMAGE_CUBEMAP) != 0;
    if (cube && width != 6 * height) return set_error(SLIM_ERR_ARGUMENT, "slimBakeTexture: a cube map is 6h x h");
    if ((uint64_t)width * height > (1ull << 28)) return set_error(SLIM_ERR_LIMIT, "slimBakeTexture: image too large");
    uint32_t f = flags & (SLIM_IMAGE_LINEAR | SLIM_IMAGE_MIPMAP | SLIM_IMAGE_WRAP | SLIM_IMAGE_NORMAL | SLIM_IMAGE_CUBEMAP);
    if (channels == 4) f |= SLIM_IMAGE_ALPHA;
    bool linear = (f & SLIM_IMAGE_LINEAR) != 0;
    std::vector<MipLoader> loaders;
    if (cube) {
        f &= ~(SLIM_IMAGE_WRAP | SLIM_IMAGE_NORMAL | SLIM_IMAGE_MIPMAP);
        uint32_t face = height, main = face * 4;
        loaders.resize(3);
        loaders[0].init(main, height);
        loaders[1].init(face, height);
        loaders[2].init(face, height);
        const uint8_t *c = bgr;
        for (uint32_t y = 0; y < height; y++)
            for (uint32_t x = 0; x < width; x++, c += channels) {
                Px p = component_pixel(c, channels, linear);
                if (x < main) loaders[0].texels[(size_t)main * y + x] = p;
                else if (x < main + face) loaders[1].texels[(size_t)height * y + (x - main)] = p;
                else loaders[2].texels[(size_t)height * y + (x - (main + face))] = p;
            }
        loaders[0].load(false, CubeMain, nullptr, loaders[1].texels.data(), loaders[2].texels.data());
        loaders[1].load(false, CubeTop, loaders[0].texels.data());
        loaders[2].load(false, CubeBottom, loaders[0].texels.data());
    } else {
        uint32_t count = 1;
        if (f & SLIM_IMAGE_MIPMAP) {
            uint32_t w = width, h = height;
            while (w > 4 && h > 4) { w /= 2; h /= 2; count++; }
        }
        loaders.resize(count);
        loaders[0].init(width, height);
        const uint8_t *c = bgr;
        for (size_t i = 0; i < (size_t)width * height; i++, c += channels)
            loaders[0].texels[i] = component_pixel(c, channels, linear);
        if (f & SLIM_IMAGE_NORMAL) {   // bmp2texture.cpp:306-321
            for (size_t i = 0; i < (size_t)width * height; i++) {
                Px &p = loaders[0].texels[i];
                float r = p.r * 2.0f - 1.0f;
                float g = p.g * 2.0f - 1.0f;
                float l_rcp = 1.0f / sqrtf(r * r + g * g + 1.0f);
                r *= l_rcp;
                g *= l_rcp;
                float b = sqrtf(1.0f - r * r - g * g);
                p.r = r * 0.5f + 0.5f;
                p.g = g * 0.5f + 0.5f;
                p.b = b * 0.5f + 0.5f;
            }
        }
        bool wrap = (f & SLIM_IMAGE_WRAP) != 0;
        loaders[0].load(wrap);
        // loadMips (bmp2texture.cpp:212-237): 2x2 box filter of the quads
        uint32_t w = width, h = height;
        for (uint32_t m = 1; m < count; m++) {
            uint32_t start = w + 1, stride = start * 2;
            w /= 2;
            h /= 2;
            MipLoader &prev = loaders[m - 1], &next = loaders[m];
            next.init(w, h);
            for (uint32_t y = 0; y < h; y++) {
                uint32_t offset = start + 1;
                for (uint32_t x = 0; x < w; x++) {
                    const PxQuad &q = prev.quads[offset];
                    Px &t = next.texels[(size_t)w * y + x];
                    t.r = 0.25f * (q.TL.r + q.TR.r + q.BL.r + q.BR.r);
                    t.g = 0.25f * (q.TL.g + q.TR.g + q.BL.g + q.BR.g);
                    t.b = 0.25f * (q.TL.b + q.TR.b + q.BL.b + q.BR.b);
                    offset += 2;
                }
                start += stride;
            }
            next.load(wrap);
        }
    }
    uint64_t total = 0;
    for (auto &l : loaders) total += l.quad_count();
    if (total > 0xFFFFFFFFull) return set_error(SLIM_ERR_LIMIT, "slimBakeTexture: too many texel quads");
    memset(texture, 0, sizeof(*texture));
    texture->width = width;
    texture->height = height;
    texture->size = width * height;
    texture->stride = width;
    texture->mip_count = (uint32_t)loaders.size();
    texture->flags = f;
    *mip_count = (uint32_t)loaders.size();
    *quad_count = (uint32_t)total;
    if (!quads || !mips) return SLIM_OK;   // sizing call
    SlimTexelQuad *q = quads;
    for (size_t m = 0; m < loaders.size(); m++) {
        MipLoader &l = loaders[m];
        mips[m].width = l.width;
        mips[m].height = l.height;
        mips[m].texel_quads = q;
        for (size_t k = 0; k < l.quad_count(); k++) {
            const PxQuad &p = l.quads[k];
            q->R[0] = to_byte(p.TL.r); q->G[0] = to_byte(p.TL.g); q->B[0] = to_byte(p.TL.b);
            q->R[1] = to_byte(p.TR.r); q->G[1] = to_byte(p.TR.g); q->B[1] = to_byte(p.TR.b);
            q->R[2] = to_byte(p.BL.r); q->G[2] = to_byte(p.BL.g); q->B[2] = to_byte(p.BL.b);
            q->R[3] = to_byte(p.BR.r); q->G[3] = to_byte(p.BR.g); q->B[3] = to_byte(p.BR.b);
            q++;
        }
    }
    texture->mips = mips;
    return SLIM_OK;
}

}  // namespace slim
