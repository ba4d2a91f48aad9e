// Headless volume ray-march of the smoke density into an RGB buffer: the
// reference's volume shader (src/renderer/shaders/volume.frag:13-55) and its
// orbit camera (src/renderer/OrbitCamera.cpp:5-28) as one CUDA thread per
// pixel, with no graphics API. The shader runs for the pixels whose ray meets
// the box (the rasteriser's back faces of the cube); its 3D texture lookup
// (linear filter, clamp to edge) is the cell-centred trilinear sample of the
// density in FP32. Pixel (i, j) counts j from the bottom row, as OpenGL does;
// pixels with no smoke keep the clear colour.
#include "engine.hpp"
#include "kernels.hpp"

#include <cmath>

namespace vb {
namespace {

struct Camera {
    float pos[3];
    float right[3], up[3], fwd[3];
    float inv_p0, inv_p5;  // 1 / projection scale in x and y
};

// buildMVP (OrbitCamera.cpp:5-28): camera on a sphere around the box centre,
// 0.8 rad vertical field of view.
Camera orbit_camera(float azimuth, float elevation, float dist, float aspect, float box) {
    Camera c;
    const float cax = cosf(azimuth), sax = sinf(azimuth), cel = cosf(elevation), sel = sinf(elevation);
    const float half = box * 0.5f;
    c.pos[0] = half + dist * cel * cax;
    c.pos[1] = half + dist * cel * sax;
    c.pos[2] = half + dist * sel;
    const float upx = -sel * cax, upy = -sel * sax, upz = cel;
    float fx = half - c.pos[0], fy = half - c.pos[1], fz = half - c.pos[2];
    const float fl = sqrtf(fx * fx + fy * fy + fz * fz);
    fx /= fl;
    fy /= fl;
    fz /= fl;
    c.right[0] = fy * upz - fz * upy;
    c.right[1] = fz * upx - fx * upz;
    c.right[2] = fx * upy - fy * upx;
    c.up[0] = upx;
    c.up[1] = upy;
    c.up[2] = upz;
    c.fwd[0] = fx;
    c.fwd[1] = fy;
    c.fwd[2] = fz;
    const float f = 1.0f / tanf(0.8f * 0.5f);
    c.inv_p0 = 1.f / (f / aspect);
    c.inv_p5 = 1.f / f;
    return c;
}

// Texture lookup at normalised coordinates (GL_LINEAR, clamp to edge):
// texel centres at (i + .5) / n.
__device__ __forceinline__ float volume_at(const float* __restrict__ d, int n, float sx, float sy, float sz) {
    const float nf = float(n);
    auto axis = [&](float s, int& i0, int& i1, float& t) {
        const float g = clampf_ref(s * nf - 0.5f, 0.f, nf - 1.f);
        i0 = int(g);
        i1 = min(i0 + 1, n - 1);
        t = g - float(i0);
    };
    int x0, x1, y0, y1, z0, z1;
    float tx, ty, tz;
    axis(sx, x0, x1, tx);
    axis(sy, y0, y1, ty);
    axis(sz, z0, z1, tz);
    auto at = [&](int x, int y, int z) { return __ldg(d + (size_t(z) * n + y) * n + x); };
    return trilinear(at(x0, y0, z0), at(x1, y0, z0), at(x0, y1, z0), at(x1, y1, z0), at(x0, y0, z1),
                     at(x1, y0, z1), at(x0, y1, z1), at(x1, y1, z1), tx, ty, tz);
}

__global__ void k_raymarch(const float* __restrict__ d, int n, float box, int width, int height, Camera cam,
                           vapor_render_params p, float* __restrict__ rgb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= width || j >= height) return;
    const float bg[3] = {0.03f, 0.04f, 0.07f};
    float* out = rgb + 3 * (size_t(j) * width + i);
    out[0] = bg[0];
    out[1] = bg[1];
    out[2] = bg[2];
    // ray through the pixel centre
    const float xn = (float(i) + 0.5f) / float(width) * 2.f - 1.f, yn = (float(j) + 0.5f) / float(height) * 2.f - 1.f;
    const float vx = xn * cam.inv_p0, vy = yn * cam.inv_p5;
    float rd[3];
    for (int k = 0; k < 3; ++k) rd[k] = cam.right[k] * vx + cam.up[k] * vy + cam.fwd[k];
    const float len = sqrtf(rd[0] * rd[0] + rd[1] * rd[1] + rd[2] * rd[2]);
    for (int k = 0; k < 3; ++k) rd[k] = rd[k] / len;
    const float* ro = cam.pos;
    float tnear = -INFINITY, tfar = INFINITY;
    for (int k = 0; k < 3; ++k) {
        const float t0 = (0.f - ro[k]) / rd[k], t1 = (box - ro[k]) / rd[k];
        tnear = fmaxf(tnear, fminf(t0, t1));
        tfar = fminf(tfar, fmaxf(t0, t1));
    }
    if (tnear < 0.f) tnear = 0.f;
    if (!(tnear < tfar)) return;
    const float step = p.step_scale / float(n);
    const float smoke[3] = {0.9f, 0.85f, 0.75f};
    float col[4] = {0.f, 0.f, 0.f, 0.f};
    bool hit = false;
    for (float t = tnear; t < tfar; t += step) {
        const float px = ro[0] + rd[0] * t, py = ro[1] + rd[1] * t, pz = ro[2] + rd[2] * t;
        const float dv = volume_at(d, n, px / box, py / box, pz / box);
        if (dv > 0.001f) {
            hit = true;
            float shadow = 1.f;
            if (p.shadow_strength > 0.f) {
                float sa = 0.f;
                for (float st = p.shadow_step; st < box * 2.f; st += p.shadow_step) {
                    const float sx = px + p.light[0] * st, sy = py + p.light[1] * st, sz = pz + p.light[2] * st;
                    if (sx < 0.f || sx > box || sy < 0.f || sy > box || sz < 0.f || sz > box) break;
                    sa += volume_at(d, n, sx / box, sy / box, sz / box) * p.shadow_step * p.alpha_mul *
                          p.shadow_strength;
                    if (sa > 3.f) break;
                }
                shadow = expf(-sa);
            }
            const float alpha = clampf_ref(dv * step * p.alpha_mul, 0.f, 1.f);
            for (int k = 0; k < 3; ++k) col[k] += (1.f - col[3]) * smoke[k] * alpha * shadow;
            col[3] += (1.f - col[3]) * alpha;
        }
        if (col[3] > 0.99f) break;
    }
    if (!hit) return;
    for (int k = 0; k < 3; ++k) out[k] = bg[k] * (1.f - col[3]) + col[k];
}

}  // namespace

void render_volume(const float* density, int n, float box, const vapor_render_params& p, float* rgb, cudaStream_t s) {
    const Camera cam = orbit_camera(p.azimuth, p.elevation, p.distance, float(p.width) / float(p.height), box);
    const dim3 block(16, 16), grid((p.width + 15) / 16, (p.height + 15) / 16);
    count_launch();
    k_raymarch<<<grid, block, 0, s>>>(density, n, box, p.width, p.height, cam, p, rgb);
    VB_CUDA(cudaGetLastError());
}

}  // namespace vb
