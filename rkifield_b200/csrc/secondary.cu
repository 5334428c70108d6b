// secondary.cu — shadow and ambient-occlusion rays from a view's G-buffer.
//
// The reference's shading pass (shade_main.wgsl, shade_common_shading.wgsl:
// 9-47) turns every hit pixel into shadow queries towards the lights and
// ambient-occlusion queries about the normal.  This kernel builds those
// queries as ray batches for the batched march: per pixel, n_lights shadow
// rays (origin = hit + normal * shadow_bias, towards each point light,
// tmax = distance to it) and ao_per_hit cosine-weighted hemisphere rays
// (origin = hit + normal * ao_bias, tmax = ao_radius).  Pixel p owns ray
// slots [p*n, p*n + n); pixels that missed get tmax = -1, which ends the ray
// on its first iteration, so the layout needs no compaction and is
// deterministic.  Directions come from a counter-based hash of
// (seed, pixel, ray), so the rays do not depend on launch order.
#include <cstring>

#include "ctx.h"

namespace rkf {
namespace detail {

__device__ __forceinline__ uint32_t hash32(uint32_t x) {
  // integer finaliser of MurmurHash3 (Appleby)
  x ^= x >> 16;
  x *= 0x85ebca6bu;
  x ^= x >> 13;
  x *= 0xc2b2ae35u;
  x ^= x >> 16;
  return x;
}

__device__ __forceinline__ float unit_float(uint32_t h) {
  return static_cast<float>(h >> 8) * (1.0f / 16777216.0f);  // [0, 1)
}

struct SecParams {
  float pos[3], fwd[3], right[3], up[3];
  uint32_t w, h;
  const float* t;
  const float* normal;
  const uint16_t* flags;
  float lights[3 * 16];
  uint32_t n_lights, ao_per_hit;
  float ao_radius, shadow_bias, ao_bias;
  uint32_t seed;
  float* so;
  float* sd;
  float* st;
  float* ao;
  float* ad;
  float* at;
  unsigned int* hits;
};

__global__ void k_secondary(SecParams k) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= k.w * k.h) return;
  const bool hit = (k.flags[i] & RKF_FLAG_HIT) != 0;
  float hx = 0, hy = 0, hz = 0, nx = 0, ny = 1, nz = 0;
  if (hit) {
    atomicAdd(k.hits, 1u);
    const uint32_t px = i % k.w, py = i / k.w;
    const float u = (static_cast<float>(px) + 0.5f) / static_cast<float>(k.w);
    const float v = (static_cast<float>(py) + 0.5f) / static_cast<float>(k.h);
    float dx = k.fwd[0] + (u * 2.0f - 1.0f) * k.right[0] + (1.0f - v * 2.0f) * k.up[0];
    float dy = k.fwd[1] + (u * 2.0f - 1.0f) * k.right[1] + (1.0f - v * 2.0f) * k.up[1];
    float dz = k.fwd[2] + (u * 2.0f - 1.0f) * k.right[2] + (1.0f - v * 2.0f) * k.up[2];
    const float il = rsqrtf(dx * dx + dy * dy + dz * dz);
    dx *= il;
    dy *= il;
    dz *= il;
    const float t = k.t[i];
    hx = k.pos[0] + dx * t;
    hy = k.pos[1] + dy * t;
    hz = k.pos[2] + dz * t;
    nx = k.normal[3 * static_cast<size_t>(i)];
    ny = k.normal[3 * static_cast<size_t>(i) + 1];
    nz = k.normal[3 * static_cast<size_t>(i) + 2];
  }
  for (uint32_t l = 0; l < k.n_lights; ++l) {
    const size_t r = static_cast<size_t>(i) * k.n_lights + l;
    const float ox = hx + nx * k.shadow_bias, oy = hy + ny * k.shadow_bias, oz = hz + nz * k.shadow_bias;
    float dx = k.lights[3 * l] - ox, dy = k.lights[3 * l + 1] - oy, dz = k.lights[3 * l + 2] - oz;
    const float len = sqrtf(dx * dx + dy * dy + dz * dz);
    const float il = len > 0.0f ? 1.0f / len : 0.0f;
    k.so[3 * r] = ox;
    k.so[3 * r + 1] = oy;
    k.so[3 * r + 2] = oz;
    k.sd[3 * r] = dx * il;
    k.sd[3 * r + 1] = dy * il;
    k.sd[3 * r + 2] = dz * il;
    k.st[r] = hit ? len : -1.0f;
  }
  // tangent frame of the normal
  const float ax = fabsf(nx) < 0.9f ? 1.0f : 0.0f, ay = fabsf(nx) < 0.9f ? 0.0f : 1.0f;
  float tx = ay * nz, ty = -ax * nz, tz = ax * ny - ay * nx;  // a x n
  const float itl = rsqrtf(fmaxf(tx * tx + ty * ty + tz * tz, 1e-20f));
  tx *= itl;
  ty *= itl;
  tz *= itl;
  const float bx = ny * tz - nz * ty, by = nz * tx - nx * tz, bz = nx * ty - ny * tx;
  for (uint32_t a = 0; a < k.ao_per_hit; ++a) {
    const size_t r = static_cast<size_t>(i) * k.ao_per_hit + a;
    const uint32_t h0 = hash32(k.seed ^ hash32(i * 0x9E3779B9u + a));
    const float r1 = unit_float(h0), r2 = unit_float(hash32(h0 ^ 0x68bc21ebu));
    const float rr = sqrtf(r1), phi = 6.28318530718f * r2;
    const float lx = rr * cosf(phi), ly = rr * sinf(phi), lz = sqrtf(fmaxf(0.0f, 1.0f - r1));
    k.ao[3 * r] = hx + nx * k.ao_bias;
    k.ao[3 * r + 1] = hy + ny * k.ao_bias;
    k.ao[3 * r + 2] = hz + nz * k.ao_bias;
    k.ad[3 * r] = lx * tx + ly * bx + lz * nx;
    k.ad[3 * r + 1] = lx * ty + ly * by + lz * ny;
    k.ad[3 * r + 2] = lx * tz + ly * bz + lz * nz;
    k.at[r] = hit ? k.ao_radius : -1.0f;
  }
}

}  // namespace detail
}  // namespace rkf

using namespace rkf;

extern "C" rkf_status rkf_secondary_rays(rkf_ctx* ctx, const rkf_camera* cam, uint32_t w, uint32_t h,
                                         const rkf_gbuffer* gb, const float* lights, uint32_t n_lights,
                                         uint32_t ao_per_hit, float ao_radius, uint32_t seed,
                                         float* shadow_o, float* shadow_d, float* shadow_tmax,
                                         float* ao_o, float* ao_d, float* ao_tmax,
                                         uint32_t* hit_pixels, void* stream) {
  if (!ctx || !cam || !gb || (n_lights && !lights) || !hit_pixels)
    return fail(RKF_INVALID_ARG, "rkf_secondary_rays: null argument");
  if (gb->mem != RKF_MEM_DEVICE || !gb->t || !gb->normal || !gb->flags)
    return fail(RKF_INVALID_ARG, "rkf_secondary_rays: device G-buffer required");
  if (n_lights > 16) return fail(RKF_INVALID_ARG, "rkf_secondary_rays: at most 16 lights");
  if ((n_lights && (!shadow_o || !shadow_d || !shadow_tmax)) || (ao_per_hit && (!ao_o || !ao_d || !ao_tmax)))
    return fail(RKF_INVALID_ARG, "rkf_secondary_rays: missing output array");
  if (w == 0 || h == 0) return fail(RKF_INVALID_ARG, "rkf_secondary_rays: empty view");
  Ctx* c = reinterpret_cast<Ctx*>(ctx);
  RKF_CUDA_TRY(cudaSetDevice(c->device));
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : c->stream;
  detail::SecParams k;
  std::memset(&k, 0, sizeof(k));
  for (int a = 0; a < 3; ++a) {
    k.pos[a] = cam->position[a];
    k.fwd[a] = cam->forward[a];
    k.right[a] = cam->right[a];
    k.up[a] = cam->up[a];
  }
  k.w = w;
  k.h = h;
  k.t = gb->t;
  k.normal = gb->normal;
  k.flags = gb->flags;
  std::memcpy(k.lights, lights, sizeof(float) * 3 * n_lights);
  k.n_lights = n_lights;
  k.ao_per_hit = ao_per_hit;
  k.ao_radius = ao_radius;
  k.shadow_bias = 0.08f;  // SHADOW_BIAS (shade_common.wgsl:276)
  k.ao_bias = 0.02f;
  k.seed = seed;
  k.so = shadow_o;
  k.sd = shadow_d;
  k.st = shadow_tmax;
  k.ao = ao_o;
  k.ad = ao_d;
  k.at = ao_tmax;
  unsigned int* dh = reinterpret_cast<unsigned int*>(c->counters.as<char>() + 256);
  RKF_CUDA_TRY(cudaMemsetAsync(dh, 0, 4, st));
  k.hits = dh;
  const uint64_t n = static_cast<uint64_t>(w) * h;
  detail::k_secondary<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(k);
  c->counted();
  RKF_CUDA_TRY(cudaGetLastError());
  RKF_CUDA_TRY(cudaMemcpyAsync(hit_pixels, dh, 4, cudaMemcpyDeviceToHost, st));
  RKF_CUDA_TRY(cudaStreamSynchronize(st));
  return RKF_OK;
}
