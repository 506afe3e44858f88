// sf_render.cu -- headless volume ray-march of one field into an RGBA image:
// the reference viewer's volume shader (vulkan-app/shaders/field_volume.slang)
// restated as a CUDA kernel, with the framebuffer replaced by a device
// buffer. One thread per pixel; the field is read by trilinear gathers
// (fields up to 512^3 stay mostly in L2 across a frame).
//
// Per pixel (field_volume.slang:122-175): a primary ray from the camera
// (perspective or orthographic, make_ray :61-79), clipped to the volume's box
// (intersect_aabb :81-97), marched in `steps` equal steps at the segment
// midpoints; each sample is the trilinear value of the field at the sample's
// box coordinates (sample_field :37-59: clamped, corner indices clamped to
// the grid), scaled, mapped to [0, 1] (a signed range maps |value| and picks
// colour A or B by sign; otherwise a linear ramp from colour A to B), and
// composited front to back with alpha = 1 - exp(-v * density * step);
// samples below 1e-4 are skipped and the march stops once transmittance is
// below 0.01. Output: premultiplied colour and alpha = 1 - transmittance.

#include <cuda_runtime.h>

#include "sf_launch.h"

namespace sfb {

namespace {

__device__ __forceinline__ float3 f3(const float* v) { return make_float3(v[0], v[1], v[2]); }
__device__ __forceinline__ float3 add3(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 mul3(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 normalize3(float3 v) {
    const float n = sqrtf(v.x * v.x + v.y * v.y + v.z * v.z);
    return make_float3(v.x / n, v.y / n, v.z / n);
}
__device__ __forceinline__ float lerpf(float a, float b, float t) { return a + t * (b - a); }
__device__ __forceinline__ float saturatef(float v) { return fminf(fmaxf(v, 0.0f), 1.0f); }
__device__ __forceinline__ float safe_dir(float d) { return fabsf(d) < 1.0e-6f ? (d < 0.0f ? -1.0e-6f : 1.0e-6f) : d; }

// sample_field: trilinear value at box coordinates uvw in [0, 1]^3.
__device__ __forceinline__ float sample_field(const float* __restrict__ f, float3 uvw, int nx, int ny, int nz) {
    uvw = make_float3(saturatef(uvw.x), saturatef(uvw.y), saturatef(uvw.z));
    const float px = uvw.x * static_cast<float>(nx - 1), py = uvw.y * static_cast<float>(ny - 1), pz = uvw.z * static_cast<float>(nz - 1);
    const float fx = floorf(px), fy = floorf(py), fz = floorf(pz);
    const int lx = static_cast<int>(fx), ly = static_cast<int>(fy), lz = static_cast<int>(fz);
    const int hx = min(lx + 1, nx - 1), hy = min(ly + 1, ny - 1), hz = min(lz + 1, nz - 1);
    const float tx = px - fx, ty = py - fy, tz = pz - fz;
    const size_t sy = static_cast<size_t>(nx), sz = static_cast<size_t>(nx) * static_cast<size_t>(ny);
    const auto at = [&](int x, int y, int z) { return __ldg(&f[static_cast<size_t>(x) + sy * static_cast<size_t>(y) + sz * static_cast<size_t>(z)]); };
    const float c00 = lerpf(at(lx, ly, lz), at(hx, ly, lz), tx);
    const float c10 = lerpf(at(lx, hy, lz), at(hx, hy, lz), tx);
    const float c01 = lerpf(at(lx, ly, hz), at(hx, ly, hz), tx);
    const float c11 = lerpf(at(lx, hy, hz), at(hx, hy, hz), tx);
    return lerpf(lerpf(c00, c10, ty), lerpf(c01, c11, ty), tz);
}

__global__ void __launch_bounds__(256) k_render_volume(const float* __restrict__ field, int nx, int ny, int nz, RenderParams p, float4* __restrict__ out) {
    const int px = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x), py = static_cast<int>(blockIdx.y * blockDim.y + threadIdx.y);
    if (px >= p.width || py >= p.height) return;
    // the fragment's NDC (pixel centre; row 0 at the top), uv = (ndc.x, -ndc.y)
    const float u = (static_cast<float>(px) + 0.5f) / static_cast<float>(p.width) * 2.0f - 1.0f;
    const float v = -((static_cast<float>(py) + 0.5f) / static_cast<float>(p.height) * 2.0f - 1.0f);
    float3 origin, dir;
    if (p.projection != 0) {
        const float hh = p.ortho_height * 0.5f, hw = hh * p.aspect;
        origin = add3(add3(f3(p.eye), mul3(f3(p.right), u * hw)), mul3(f3(p.up), v * hh));
        dir = normalize3(f3(p.forward));
    } else {
        origin = f3(p.eye);
        dir = normalize3(add3(add3(f3(p.forward), mul3(f3(p.right), u * p.aspect * p.tan_half_fov)), mul3(f3(p.up), v * p.tan_half_fov)));
    }
    const float3 bmin = f3(p.volume_min), bmax = f3(p.volume_max);
    const float3 inv = make_float3(1.0f / safe_dir(dir.x), 1.0f / safe_dir(dir.y), 1.0f / safe_dir(dir.z));
    const float3 t0v = make_float3((bmin.x - origin.x) * inv.x, (bmin.y - origin.y) * inv.y, (bmin.z - origin.z) * inv.z);
    const float3 t1v = make_float3((bmax.x - origin.x) * inv.x, (bmax.y - origin.y) * inv.y, (bmax.z - origin.z) * inv.z);
    const float entry = fmaxf(fmaxf(fminf(t0v.x, t1v.x), fminf(t0v.y, t1v.y)), fminf(t0v.z, t1v.z));
    const float exit = fminf(fminf(fmaxf(t0v.x, t1v.x), fmaxf(t0v.y, t1v.y)), fmaxf(t0v.z, t1v.z));
    const float t0 = fmaxf(entry, 0.0f), t1 = exit;
    const size_t o = static_cast<size_t>(py) * static_cast<size_t>(p.width) + static_cast<size_t>(px);
    if (t1 <= t0) {
        out[o] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        return;
    }
    const unsigned steps = p.steps > 0u ? p.steps : 1u;
    const float step_len = (t1 - t0) / static_cast<float>(steps);
    const float3 extent = make_float3(fmaxf(bmax.x - bmin.x, 1.0e-5f), fmaxf(bmax.y - bmin.y, 1.0e-5f), fmaxf(bmax.z - bmin.z, 1.0e-5f));
    const float vmin = p.value_min, vmax = fmaxf(p.value_max, vmin + 1.0e-5f);
    const bool signed_range = vmin < 0.0f && vmax > 0.0f;
    const float abs_max = fmaxf(fabsf(vmin), fabsf(vmax));
    float trans = 1.0f;
    float3 color = make_float3(0.0f, 0.0f, 0.0f);
    for (unsigned i = 0; i < steps; ++i) {
        const float travel = t0 + (static_cast<float>(i) + 0.5f) * step_len;
        const float3 w = add3(origin, mul3(dir, travel));
        const float3 uvw = make_float3((w.x - bmin.x) / extent.x, (w.y - bmin.y) / extent.y, (w.z - bmin.z) / extent.z);
        const float value = sample_field(field, uvw, nx, ny, nz) * p.value_scale;
        float level;
        float3 sample;
        if (signed_range) {
            level = abs_max > 1.0e-5f ? saturatef(fabsf(value) / abs_max) : 0.0f;
            sample = value < 0.0f ? f3(p.color_a) : f3(p.color_b);
        } else {
            level = saturatef((value - vmin) / (vmax - vmin));
            sample = make_float3(lerpf(p.color_a[0], p.color_b[0], level), lerpf(p.color_a[1], p.color_b[1], level), lerpf(p.color_a[2], p.color_b[2], level));
        }
        if (level < 1.0e-4f) continue;
        const float alpha = 1.0f - expf(-level * p.density * step_len);
        color = add3(color, mul3(sample, trans * alpha));
        trans *= 1.0f - alpha;
        if (trans < 0.01f) break;
    }
    out[o] = make_float4(color.x, color.y, color.z, 1.0f - trans);
}

}  // namespace

cudaError_t launch_render_volume(const float* field, Dims d, const RenderParams& p, float* out_rgba, cudaStream_t s) {
    const dim3 block(16, 16);
    const dim3 grid(static_cast<unsigned>((p.width + 15) / 16), static_cast<unsigned>((p.height + 15) / 16));
    k_render_volume<<<grid, block, 0, s>>>(field, d.nx, d.ny, d.nz, p, reinterpret_cast<float4*>(out_rgba));
    return cudaGetLastError();
}

}  // namespace sfb
