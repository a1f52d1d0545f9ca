// Path shading: material dispatch, next-event estimation with MIS over
// emissive triangles, punctual lights and the importance-sampled HDR
// environment, dielectric/glossy/diffuse continuation, Russian roulette.
//
// Every function restates its reference counterpart (cited) with the same
// operation order and the same RNG draw order; elementary functions come from
// wf_math.h.  Shadow tests are routed through a Sink:
//   * DeferredSink (wavefront kernels) queues the shadow ray and records the
//     contribution as a term conditional on it; the finalize kernel adds the
//     terms in program order once visibility is known, so the radiance sum is
//     formed in the reference's order.
//   * InlineSink (persistent kernel) traces the shadow ray immediately, like
//     the reference's shadePersistentPath.
// RNG consumption never depends on visibility in the reference, which is what
// makes the deferral exact.
#pragma once

#include "wf_traverse.cuh"

namespace wf {

constexpr float kInvPi = 0.31830988618f;
constexpr float kPiF = 3.14159265359f;

// ------------------------------------------------------------------- RNG
// include/core/rng.cuh:7-51, src/core/rng.cu:4-42.
WF_HDI uint64_t split_mix64(uint64_t value) {
    value += 0x9e3779b97f4a7c15ull;
    value = (value ^ (value >> 30)) * 0xbf58476d1ce4e5b9ull;
    value = (value ^ (value >> 27)) * 0x94d049bb133111ebull;
    return value ^ (value >> 31);
}
WF_HDI uint64_t make_rng_state(uint64_t key, uint32_t strategy) {
    if (strategy == 0) {
        uint32_t seed = uint32_t(key) * 747796405u + 2891336453u;
        return seed == 0 ? 1u : seed;
    }
    return split_mix64(key);
}
WF_HDI uint64_t pixel_rng_key(uint32_t pixel, uint32_t sample, uint32_t strategy) {
    if (strategy == 0) return uint64_t(pixel ^ (sample * 0x9e3779b9u));
    return (uint64_t(sample) << 32) | pixel;
}
WF_HDI uint64_t photon_rng_key(uint32_t photon, uint32_t seed, uint32_t strategy) {
    if (strategy == 0) return uint64_t(seed ^ (photon * 0x9e3779b9u));
    return (uint64_t(seed) << 32) | photon;
}
WF_HDI float random_float(uint64_t& state, uint32_t strategy) {
    uint32_t value;
    if (strategy == 0) {
        uint32_t x = uint32_t(state);
        x ^= x << 13;
        x ^= x >> 17;
        x ^= x << 5;
        state = x;
        value = x;
    } else {
        uint64_t old = state;
        state = old * 6364136223846793005ull + 1442695040888963407ull;
        uint32_t xorshifted = uint32_t(((old >> 18u) ^ old) >> 27u);
        uint32_t rotation = uint32_t(old >> 59u);
        value = (xorshifted >> rotation) | (xorshifted << ((32u - rotation) & 31u));
    }
    return float(value >> 8) * 0x1.0p-24f;
}

// ----------------------------------------------------------------- path
struct Path {
    V3 origin, direction, throughput;
    uint32_t pixel, depth;
    uint64_t rng;
    uint32_t medium;
    float medium_density;
    float prev_pdf;
    float eta_scale;
    bool specular;
    bool active;
};

// addPathRadiance clamp, include/renderer/path_state.cuh:33-43: the clamped
// contribution (the sum itself happens in the sink).
WF_DEV V3 clamp_contribution(const Path& path, V3 c, float clamp, bool emission_or_background) {
    bool indirect = path.depth > (emission_or_background ? 1u : 0u);
    if (indirect && clamp > 0.0f) {
        float magnitude = (fabsf(c.x) / 3.0f + fabsf(c.y) / 3.0f + fabsf(c.z) / 3.0f);
        if (magnitude > clamp) c *= clamp / magnitude;
    }
    return c;
}

// -------------------------------------------------------- BSDF helpers
// include/renderer/device_sampling.cuh:6-93.
WF_DEV V3 sample_cosine_hemisphere(V3 n, Path& path, uint32_t strategy) {
    constexpr float two_pi = 6.28318530718f;
    float u1 = random_float(path.rng, strategy);
    float u2 = random_float(path.rng, strategy);
    float radius = sqrtf(u1);
    float phi = two_pi * u2;
    float x = radius * wfm::cosf(phi);
    float y = radius * wfm::sinf(phi);
    float z = sqrtf(1.0f - u1);
    V3 helper = fabsf(n.x) > 0.1f ? V3{0.0f, 1.0f, 0.0f} : V3{1.0f, 0.0f, 0.0f};
    V3 tangent = normalize(cross(helper, n));
    V3 bitangent = cross(n, tangent);
    return normalize(tangent * x + bitangent * y + n * z);
}

// randomInUnitSphere (device_sampling.cuh:27-35).  The reference builds the
// point with Vec3(r(), r(), r()), whose argument order C++ leaves unspecified;
// draws are taken x, y, z here.  Acceptance and the draw count are symmetric in
// the order, and the only caller scales the point by a roughness <= 0.
WF_DEV V3 random_in_unit_sphere(Path& path, uint32_t strategy) {
    for (;;) {
        float x = 2.0f * random_float(path.rng, strategy) - 1.0f;
        float y = 2.0f * random_float(path.rng, strategy) - 1.0f;
        float z = 2.0f * random_float(path.rng, strategy) - 1.0f;
        V3 p{x, y, z};
        if (length_squared(p) < 1.0f) return p;
    }
}

WF_DEV V3 reflect(V3 i, V3 n) { return i - 2.0f * dot(i, n) * n; }

WF_DEV V3 refract(V3 i, V3 n, float eta) {
    float cos_theta = fminf(dot(-i, n), 1.0f);
    V3 perpendicular = eta * (i + cos_theta * n);
    V3 parallel = -sqrtf(fmaxf(0.0f, 1.0f - length_squared(perpendicular))) * n;
    return perpendicular + parallel;
}

WF_DEV float dielectric_reflectance(float cosine, float eta) {
    if (eta == 1.0f) return 0.0f;
    cosine = fminf(1.0f, fmaxf(0.0f, cosine));
    float sin2t = eta * eta * fmaxf(0.0f, 1.0f - cosine * cosine);
    if (sin2t >= 1.0f) return 1.0f;
    float cos_t = sqrtf(1.0f - sin2t);
    float perpendicular = (eta * cosine - cos_t) / (eta * cosine + cos_t);
    float parallel = (cosine - eta * cos_t) / (cosine + eta * cos_t);
    return 0.5f * (perpendicular * perpendicular + parallel * parallel);
}

struct DielectricInterface {
    V3 normal, reflection, transmission;
    float eta, reflectance;
    bool front_face;
};

WF_CALL DielectricInterface dielectric_interface(V3 incident, V3 geometric, V3 shading, float ior) {
    bool front = dot(incident, geometric) < 0.0f;
    V3 facing = front ? geometric : -geometric;
    if (dot(shading, geometric) < 0.0f) shading = -shading;
    V3 normal = front ? shading : -shading;
    float eta = front ? 1.0f / ior : ior;
    if (dot(incident, normal) >= 0.0f) normal = facing;
    float reflectance = dielectric_reflectance(dot(-incident, normal), eta);
    V3 reflection = reflect(incident, normal);
    V3 transmission = refract(incident, normal, eta);
    if (dot(reflection, facing) <= 0.0f || (reflectance < 1.0f && dot(transmission, facing) >= 0.0f)) {
        normal = facing;
        reflectance = dielectric_reflectance(dot(-incident, normal), eta);
        reflection = reflect(incident, normal);
        transmission = refract(incident, normal, eta);
    }
    return DielectricInterface{normal, reflection, transmission, eta, reflectance, front};
}

// include/renderer/specular_glossiness.cuh:7-80.
struct SpecGloss {
    V3 diffuse, f0;
    float roughness;
};
WF_DEV float sg_max(V3 v) { return fmaxf(v.x, fmaxf(v.y, v.z)); }
WF_DEV float sg_probability(const SpecGloss& s) {
    float specular = sg_max(s.f0);
    float diffuse = sg_max(s.diffuse) * (1.0f - specular);
    return fminf(0.95f, fmaxf(0.05f, specular / fmaxf(1.0e-6f, specular + diffuse)));
}
WF_DEV float sg_alpha(const SpecGloss& s) {
    float r = fmaxf(0.02f, s.roughness);
    return r * r;
}
WF_DEV float sg_d(float nh, float alpha) {
    float a2 = alpha * alpha;
    float den = (1.0f - nh * nh) + a2 * nh * nh;
    return a2 / (kPiF * den * den);
}
WF_DEV float sg_g1(float cosine, float alpha) {
    return 2.0f * cosine / (cosine + sqrtf(alpha * alpha + (1.0f - alpha * alpha) * cosine * cosine));
}
WF_CALL V3 sg_evaluate(const SpecGloss& s, V3 n, V3 outgoing, V3 incoming, float& pdf) {
    pdf = 0.0f;
    float nv = dot(n, outgoing), nl = dot(n, incoming);
    V3 sum = outgoing + incoming;
    if (nv <= 0.0f || nl <= 0.0f || length_squared(sum) < 1.0e-12f) return V3{0, 0, 0};
    V3 half = normalize(sum);
    float nh = fminf(1.0f, fmaxf(0.0f, dot(n, half)));
    float vh = fminf(1.0f, fmaxf(1.0e-8f, dot(outgoing, half)));
    float alpha = sg_alpha(s);
    float d = sg_d(nh, alpha);
    float probability = sg_probability(s);
    pdf = (1.0f - probability) * nl * kInvPi + probability * d * nh / (4.0f * vh);
    float schlick = wfm::powf(1.0f - vh, 5.0f);
    V3 fresnel = s.f0 + (V3{1.0f, 1.0f, 1.0f} - s.f0) * schlick;
    V3 diffuse = s.diffuse * ((1.0f - sg_max(s.f0)) * kInvPi);
    float g = sg_g1(nv, alpha) * sg_g1(nl, alpha);
    return diffuse + fresnel * (d * g / (4.0f * nv * nl));
}
WF_DEV V3 sg_basis(V3 n, float x, float y, float z) {
    V3 helper = fabsf(n.x) > 0.1f ? V3{0.0f, 1.0f, 0.0f} : V3{1.0f, 0.0f, 0.0f};
    V3 tangent = normalize(cross(helper, n));
    return normalize(x * tangent + y * cross(n, tangent) + z * n);
}
WF_DEV V3 sg_sample(const SpecGloss& s, V3 n, V3 outgoing, float choice, float u, float v) {
    float phi = 6.28318530718f * v;
    if (choice < sg_probability(s)) {
        float alpha = sg_alpha(s);
        float cosine = sqrtf((1.0f - u) / (1.0f + (alpha * alpha - 1.0f) * u));
        float sine = sqrtf(fmaxf(0.0f, 1.0f - cosine * cosine));
        V3 half = sg_basis(n, sine * wfm::cosf(phi), sine * wfm::sinf(phi), cosine);
        return 2.0f * dot(outgoing, half) * half - outgoing;
    }
    float radius = sqrtf(u);
    return sg_basis(n, radius * wfm::cosf(phi), radius * wfm::sinf(phi), sqrtf(1.0f - u));
}

// include/renderer/gltf_pbr.cuh:8-119.
struct GltfPbr {
    V3 color, normal, coat_normal;
    float metallic, roughness;
    V3 dielectric_f0;
    float dielectric_f90;
    float coat, coat_roughness;
    V3 reflection_normal;
};
struct GltfWeights {
    float diffuse, specular, coat;
};
WF_DEV V3 gltf_reflection_normal(V3 normal, V3 geometric, V3 view) {
    float gv = dot(geometric, view);
    if (gv <= 0.f) return geometric;
    float target = fminf(.01f, .9f * gv);
    V3 reflected = 2.f * dot(normal, view) * normal - view;
    if (dot(geometric, reflected) >= target) return normal;
    float lower = 0.f, upper = 1.f;
#pragma unroll 1
    for (int i = 0; i < 24; ++i) {
        float t = (lower + upper) * .5f;
        V3 candidate = normalize(normal * (1.f - t) + geometric * t);
        reflected = 2.f * dot(candidate, view) * candidate - view;
        if (dot(geometric, reflected) >= target) upper = t; else lower = t;
    }
    return normalize(normal * (1.f - upper) + geometric * upper);
}
WF_DEV V3 pbr_specular_normal(const GltfPbr& s) {
    return length_squared(s.reflection_normal) > 0.f ? s.reflection_normal : s.normal;
}
WF_DEV void correct_gltf_normals(GltfPbr& s, V3 geometric, V3 view) {
    s.reflection_normal = gltf_reflection_normal(s.normal, geometric, view);
    if (s.coat > 0.f) s.coat_normal = gltf_reflection_normal(s.coat_normal, geometric, view);
}
WF_DEV float pbr_saturate(float x) { return fminf(1.f, fmaxf(0.f, x)); }
WF_DEV float pbr_schlick(float cosine) {
    float x = 1.f - pbr_saturate(cosine);
    return x * x * x * x * x;
}
WF_DEV float pbr_coat_weight(const GltfPbr& s, V3 view) {
    return s.coat * (.04f + .96f * pbr_schlick(dot(s.coat_normal, view)));
}
WF_DEV V3 pbr_dielectric_fresnel(const GltfPbr& s, float cosine) {
    return s.dielectric_f0 +
           (V3{s.dielectric_f90, s.dielectric_f90, s.dielectric_f90} - s.dielectric_f0) * pbr_schlick(cosine);
}
WF_DEV V3 pbr_base_fresnel(const GltfPbr& s, float cosine) {
    V3 metal = s.color + (V3{1, 1, 1} - s.color) * pbr_schlick(cosine);
    return pbr_dielectric_fresnel(s, cosine) * (1.f - s.metallic) + metal * s.metallic;
}
WF_DEV GltfWeights pbr_weights(const GltfPbr& s, V3 view) {
    float coat = pbr_coat_weight(s, view);
    float specular = s.metallic + (1.f - s.metallic) * sg_max(pbr_dielectric_fresnel(s, dot(pbr_specular_normal(s), view)));
    return GltfWeights{(1.f - coat) * (1.f - specular), (1.f - coat) * specular, coat};
}
WF_DEV float pbr_alpha(float roughness) { return fmaxf(1.e-4f, roughness * roughness); }
WF_DEV float pbr_reflection_pdf(V3 normal, V3 view, V3 light, float roughness) {
    if (roughness <= 0 || dot(normal, view) <= 0 || dot(normal, light) <= 0 || length_squared(view + light) < 1.e-12f)
        return 0;
    V3 half = normalize(view + light);
    float vh = dot(view, half), nh = dot(normal, half);
    return vh > 0 && nh > 0 ? sg_d(pbr_saturate(nh), pbr_alpha(roughness)) * nh / (4.f * vh) : 0.f;
}
WF_DEV float pbr_reflection_kernel(V3 normal, V3 view, V3 light, float roughness) {
    float nv = dot(normal, view), nl = dot(normal, light);
    if (roughness <= 0 || nv <= 0 || nl <= 0 || length_squared(view + light) < 1.e-12f) return 0;
    float alpha = pbr_alpha(roughness), nh = pbr_saturate(dot(normal, normalize(view + light)));
    return sg_d(nh, alpha) * sg_g1(nv, alpha) * sg_g1(nl, alpha) / (4.f * nv * nl);
}
WF_DEV V3 pbr_sample_reflection(V3 normal, V3 view, float roughness, float u, float v) {
    if (roughness <= 0) return 2.f * dot(normal, view) * normal - view;
    float alpha = pbr_alpha(roughness);
    float cosine = sqrtf((1.f - u) / ((1.f - u) + alpha * alpha * u));
    float sine = sqrtf(fmaxf(0.f, 1.f - cosine * cosine)), phi = 6.28318530718f * v;
    V3 half = sg_basis(normal, sine * wfm::cosf(phi), sine * wfm::sinf(phi), cosine);
    return 2.f * dot(view, half) * half - view;
}
WF_CALL V3 pbr_evaluate_cos(const GltfPbr& s, V3 view, V3 light, float diffuse_pdf, float& pdf) {
    GltfWeights w = pbr_weights(s, view);
    float nl = fmaxf(0.f, dot(s.normal, light));
    V3 reflection_normal = pbr_specular_normal(s);
    pdf = w.diffuse * diffuse_pdf + w.specular * pbr_reflection_pdf(reflection_normal, view, light, s.roughness) +
          w.coat * pbr_reflection_pdf(s.coat_normal, view, light, s.coat_roughness);
    V3 base{0, 0, 0};
    if (length_squared(view + light) > 1.e-12f) {
        float vh = pbr_saturate(dot(view, normalize(view + light)));
        float diffuse_weight = (1.f - s.metallic) * (1.f - sg_max(pbr_dielectric_fresnel(s, vh)));
        if (dot(s.normal, view) > 0) base = s.color * (diffuse_weight * nl * .31830988618f);
        float specular_cos = fmaxf(0.f, dot(reflection_normal, light));
        base += pbr_base_fresnel(s, vh) * (pbr_reflection_kernel(reflection_normal, view, light, s.roughness) * specular_cos);
    }
    float coat_cos = fmaxf(0.f, dot(s.coat_normal, light));
    float coat_value = w.coat * pbr_reflection_kernel(s.coat_normal, view, light, s.coat_roughness) * coat_cos;
    return base * (1.f - w.coat) + V3{coat_value, coat_value, coat_value};
}

// ---------------------------------------------------------- environment
// include/scene/environment.cuh:17-71, device_traversal.cuh:571-575.
WF_DEV V3 rotate_env(V3 d, float c, float s) {
    return V3{c * d.x + s * d.z, d.y, -s * d.x + c * d.z};
}
WF_DEV void environment_uv(const Environment& e, V3 world, float& u, float& v) {
    V3 d = rotate_env(world, e.cos_neg, e.sin_neg);
    u = wfm::atan2f(d.z, d.x) / (2.0f * kPiF) + 0.5f;
    u -= floorf(u);
    float vv = wfm::atan2f(sqrtf(d.x * d.x + d.z * d.z), d.y) / kPiF;
    v = fminf(1.0f, fmaxf(0.0f, vv));
}
WF_CALL float environment_pdf(const Environment& e, V3 direction) {
    if (e.width == 0 || e.height == 0 || e.probabilities == nullptr) return 0.0f;
    float u, v;
    environment_uv(e, direction, u, v);
    uint32_t x = uint32_t(u * e.width);
    uint32_t y = uint32_t(v * e.height);
    uint32_t index = (y < e.height ? y : e.height - 1) * e.width + (x < e.width ? x : e.width - 1);
    return e.probabilities[index] / e.row_solid_angle[index / e.width];
}
// Bilinear lookup: normalized coordinates, wrap in u, clamp in v, weights
// (1-f, f), rows then columns (the texture of scene.cu:318-328 with the
// filter arithmetic of the reference's CPU replay, cpu_replay.cpp:14-24).
WF_CALL V3 environment_texel(const Environment& e, float u, float v) {
    float tx = u * e.width - .5f, ty = v * e.height - .5f;
    int x = int(floorf(tx)), y = int(floorf(ty));
    float fx = tx - x, fy = ty - y;
    float rx = 0.f, ry = 0.f, rz = 0.f;
    int w = int(e.width), h = int(e.height);
    for (int j = 0; j < 2; ++j)
        for (int i = 0; i < 2; ++i) {
            int xx = ((x + i) % w + w) % w;
            int yy = min(max(y + j, 0), h - 1);
            float4 p = __ldg(&e.pixels[size_t(yy) * e.width + xx]);
            float wt = (i ? fx : 1 - fx) * (j ? fy : 1 - fy);
            rx += wt * p.x;
            ry += wt * p.y;
            rz += wt * p.z;
        }
    return V3{rx, ry, rz};
}
WF_CALL V3 environment_radiance(const Environment& e, V3 direction) {
    float u, v;
    environment_uv(e, direction, u, v);
    return environment_texel(e, u, v) * e.intensity;
}
struct EnvSample {
    V3 direction;
    float pdf;
};
WF_CALL EnvSample sample_environment(const Environment& e, double candidate, float coin, float longitude,
                                    float latitude) {
    constexpr double pi = 3.14159265358979323846;
    uint32_t count = e.width * e.height;
    uint32_t index = uint32_t(candidate * count);
    if (index >= count) index = count - 1;
    float2 alias = __ldg(&e.alias[index]);
    if (coin >= alias.x) index = __float_as_uint(alias.y);
    uint32_t x = index % e.width, y = index / e.width;
    double u = (x + fminf(1.0f - 1.0e-7f, fmaxf(1.0e-7f, longitude))) / e.width;
    double jitter = fminf(1.0f - 1.0e-7f, fmaxf(1.0e-7f, latitude));
    double cosine = (1.0 - jitter) * wfm::cos(pi * y / e.height) + jitter * wfm::cos(pi * (y + 1.0) / e.height);
    double sine = sqrt(fmax(0.0, 1.0 - cosine * cosine));
    double phi = (u - 0.5) * 2 * pi;
    V3 local{float(sine * wfm::cos(phi)), float(cosine), float(sine * wfm::sin(phi))};
    return EnvSample{rotate_env(local, e.cos_rot, e.sin_rot), e.probabilities[index] / e.row_solid_angle[y]};
}

// ---------------------------------------------------------------- shading
WF_DEV float power_heuristic(float a, float b) {
    float a2 = a * a;
    float b2 = b * b;
    return a2 / (a2 + b2);
}

WF_DEV float diffuse_continuation_pdf(const DeviceScene& s, V3 normal, V3 direction) {
    float probability = s.env.sampling ? 0.5f : 0.0f;
    float cosine_pdf = fmaxf(0.0f, dot(normal, direction)) * 0.31830988618f;
    return probability > 0.0f ? (1.0f - probability) * cosine_pdf + probability * environment_pdf(s.env, direction)
                              : cosine_pdf;
}

WF_DEV EnvSample sample_path_environment(const DeviceScene& s, Path& path, uint32_t strategy) {
    float coarse = random_float(path.rng, strategy);
    float fine = random_float(path.rng, strategy);
    double candidate = double(coarse) + double(fine) * (1.0 / 16777216.0);
    float coin = random_float(path.rng, strategy);
    float u = random_float(path.rng, strategy);
    float v = random_float(path.rng, strategy);
    return sample_environment(s.env, candidate, coin, u, v);
}

WF_DEV float material_roughness(const Material& m) {
    return (m.flags & kMatSpecGlossWorkflow) ? 1.0f - m.glossiness : m.roughness;
}

// Hit as seen by the shading functions (hit / shadedHit of the reference).
// coat_normal: the clearcoat normal of getGltfPbrSurface before its flip
// (the hit's shading normal unless a clearcoat normal map applies).
struct ShadeHit {
    float t;
    V3 position, geometric_normal, normal;
    uint32_t material, light;
    V3 coat_normal;
};

// ------------------------------------------------------- textured materials
// srgbToLinear / gltfSrgbChannel, device_traversal.cuh:349-362.
WF_DEV V3 srgb_to_linear(float4 t) {
    return V3{wfm::powf(t.x, 2.2f), wfm::powf(t.y, 2.2f), wfm::powf(t.z, 2.2f)};
}
WF_DEV float gltf_srgb_channel(float value) {
    return value <= 0.04045f ? value / 12.92f : wfm::powf((value + 0.055f) / 1.055f, 2.4f);
}
WF_DEV V3 gltf_srgb_to_linear(float4 t) {
    return V3{gltf_srgb_channel(t.x), gltf_srgb_channel(t.y), gltf_srgb_channel(t.z)};
}

// The factors of a textured material at a hit: getMaterialAlbedo, Emission,
// Metallic, Roughness (device_traversal.cuh:363-395), getSpecGlossSurface's
// specular (:397-401), getGltfPbrSurface's specular weight and colour and
// clearcoat factors (:500-516) and getMaterialThickness (:443-449), each
// evaluated once.  Without a binding every one of them returns the factor
// itself (texel fallback 1, srgb(1) = 1), which is what untextured
// materials use directly.
WF_CALL Material resolve_material(const DeviceScene& s, const Material& m, uint32_t index, const SurfaceHit& sh) {
    const MaterialTextures& mt = s.material_textures[index];
    const float4 one = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
    Material r = m;
    bool sg = (m.flags & kMatSpecGlossWorkflow) != 0;
    float4 albedo = sample_binding(s, mt.slot[kTexAlbedo], sh.uv, sh.uv1, one);
    r.albedo = hadamard(m.albedo, sg ? gltf_srgb_to_linear(albedo) : srgb_to_linear(albedo));
    r.emission = hadamard(m.emission, srgb_to_linear(sample_binding(s, mt.slot[kTexEmissive], sh.uv, sh.uv1, one)));
    float4 mr = sample_binding(s, mt.slot[kTexMetallicRoughness], sh.uv, sh.uv1, one);
    float4 sgt = sample_binding(s, mt.slot[kTexSpecGloss], sh.uv, sh.uv1, one);
    r.metallic = m.metallic * mr.z;
    if (sg)
        r.glossiness = m.glossiness * sgt.w;  // material_roughness: 1 - glossiness * texel.w
    else
        r.roughness = m.roughness * mr.y;
    r.specular = hadamard(m.specular, gltf_srgb_to_linear(sgt));
    r.specular_weight = m.specular_weight * sample_binding(s, mt.slot[kTexSpecularWeight], sh.uv, sh.uv1, one).w;
    r.specular_color = hadamard(m.specular_color,
                                gltf_srgb_to_linear(sample_binding(s, mt.slot[kTexSpecularColor], sh.uv, sh.uv1, one)));
    r.clearcoat = m.clearcoat * sample_binding(s, mt.slot[kTexClearcoat], sh.uv, sh.uv1, one).x;
    r.clearcoat_roughness =
        m.clearcoat_roughness * sample_binding(s, mt.slot[kTexClearcoatRoughness], sh.uv, sh.uv1, one).y;
    const TexBinding& th = mt.slot[kTexThickness];
    float thickness = th.texture == kInvalid || th.texture >= s.texture_count
                          ? 1.0f
                          : sample_binding(s, th, sh.uv, sh.uv1, one).x;
    r.volume_density = m.volume_density * thickness;
    return r;
}

WF_DEV bool finite3(V3 v) { return isfinite(v.x) && isfinite(v.y) && isfinite(v.z); }

// getMaterialNormal, device_traversal.cuh:451-499: the normal map in the
// hit's tangent frame (the clearcoat normal map with its own scale for
// getGltfPbrSurface), or the hit's shading normal.
WF_CALL V3 material_normal(const DeviceScene& s, const TexBinding& b, float normal_scale, const SurfaceHit& sh) {
    if (!s.use_normal_maps || b.texture == kInvalid || b.texture >= s.texture_count) return sh.normal;
    V3 tangent = b.texcoord == 1 ? sh.tangent1 : sh.tangent;
    V3 bitangent = b.texcoord == 1 ? sh.bitangent1 : sh.bitangent;
    if (!finite3(tangent) || !finite3(bitangent) || length_squared(tangent) < 0.00000001f ||
        length_squared(bitangent) < 0.00000001f)
        return sh.normal;
    tangent = normalize(tangent - sh.normal * dot(sh.normal, tangent));
    bitangent = normalize(cross(sh.normal, tangent));
    if (!finite3(tangent) || !finite3(bitangent)) return sh.normal;
    if (dot(bitangent, b.texcoord == 1 ? sh.bitangent1 : sh.bitangent) < 0.0f) bitangent = -bitangent;
    float4 texel = sample_binding(s, b, sh.uv, sh.uv1, make_float4(0.5f, 0.5f, 1.0f, 1.0f));
    V3 tn{(texel.x * 2.0f - 1.0f) * normal_scale, (texel.y * 2.0f - 1.0f) * normal_scale, texel.z * 2.0f - 1.0f};
    tn = normalize(tn);
    if (s.normal_map_min_cosine > 0.0f && tn.z < s.normal_map_min_cosine) {
        float minimum_cosine = fminf(s.normal_map_min_cosine, 1.0f);
        float tangent_length = sqrtf(fmaxf(0.0f, tn.x * tn.x + tn.y * tn.y));
        if (tangent_length > 0.0f) {
            float scale = sqrtf(fmaxf(0.0f, 1.0f - minimum_cosine * minimum_cosine)) / tangent_length;
            tn.x *= scale;
            tn.y *= scale;
        } else {
            tn.x = 0.0f;
            tn.y = 0.0f;
        }
        tn.z = minimum_cosine;
    }
    V3 normal = tangent * tn.x + bitangent * tn.y + sh.normal * tn.z;
    if (!finite3(normal) || length_squared(normal) < 0.00000001f) return sh.normal;
    return normalize(normal);
}

// evaluateSurface, device_traversal.cuh:427-441.
WF_CALL V3 evaluate_surface(const DeviceScene& s, const Material& m, const ShadeHit& hit, V3 outgoing, V3 incoming,
                           float& pdf) {
    if (m.type == kSpecGloss)
        return sg_evaluate(SpecGloss{m.albedo, m.specular, material_roughness(m)}, hit.normal, outgoing, incoming, pdf);
    uint32_t effective = m.type == kDiffuse && m.metallic > 0.5f ? uint32_t(kMetal) : m.type;
    if (effective == kMetal) {
        if (material_roughness(m) <= 0.0f) {
            pdf = 0.0f;
            return V3{0, 0, 0};
        }
        return sg_evaluate(SpecGloss{V3{0, 0, 0}, m.albedo, material_roughness(m)}, hit.normal, outgoing, incoming, pdf);
    }
    pdf = diffuse_continuation_pdf(s, hit.normal, incoming);
    return m.albedo * 0.31830988618f;
}

// getGltfPbrSurface, device_traversal.cuh:500-516 (texture factors resolved
// by resolve_material, the clearcoat normal by shade_path).
WF_CALL GltfPbr gltf_surface(const Material& m, const ShadeHit& hit, const ShadeHit& shaded) {
    float weight = m.specular_weight;
    V3 color = m.specular_color;
    float f0 = (m.ior - 1.f) / (m.ior + 1.f);
    f0 *= f0;
    V3 df0{fminf(1.f, f0 * color.x) * weight, fminf(1.f, f0 * color.y) * weight, fminf(1.f, f0 * color.z) * weight};
    V3 coat_normal = shaded.coat_normal;
    if (dot(coat_normal, hit.geometric_normal) < 0) coat_normal = -coat_normal;
    GltfPbr g;
    g.color = m.albedo;
    g.normal = shaded.normal;
    g.coat_normal = coat_normal;
    g.metallic = m.metallic;
    g.roughness = material_roughness(m);
    g.dielectric_f0 = df0;
    g.dielectric_f90 = weight;
    g.coat = m.clearcoat;
    g.coat_roughness = m.clearcoat_roughness;
    g.reflection_normal = V3{0, 0, 0};
    return g;
}

// evaluateSurfaceCos, device_traversal.cuh:519-527.
WF_CALL V3 evaluate_surface_cos(const DeviceScene& s, const Material& m, const ShadeHit& hit, const ShadeHit& shaded,
                               V3 view, V3 light, float& pdf) {
    if (m.flags & kMatGltfPbr) {
        GltfPbr g = gltf_surface(m, hit, shaded);
        correct_gltf_normals(g, hit.geometric_normal, view);
        return pbr_evaluate_cos(g, view, light, diffuse_continuation_pdf(s, g.normal, light), pdf);
    }
    return evaluate_surface(s, m, shaded, view, light, pdf) * fmaxf(0.f, dot(shaded.normal, light));
}

// ------------------------------------------------------------------ sinks
constexpr int kMaxTerms = 8;     // per shading event
constexpr int kUnconditional = -1;

// One shading event's effect on a path: the shadow tests it needs, the
// radiance terms (each optionally conditional on one test being unoccluded)
// in the order the reference adds them, and the test (if any) whose
// unoccluded result ends the path (a terminal branch that escaped).
// Tally: the traversal variant of the shadow rays (Opaque<NoTally> when no
// material of the scene is alpha-textured).
template <typename Tally = NoTally>
struct InlineSink {
    static constexpr bool kDeferredGather = false;  // caustic gathers run inline
    const DeviceScene* scene;
    V3 radiance;
    bool killed;
    uint32_t requests;
    // Returns a handle: 1 = occluded, 0 = visible.
    WF_DEV int request(V3 o, V3 d, float t_max) {
        ++requests;
        Tally tally;
        return trace_any(*scene, o, d, t_max, tally) ? 1 : 0;
    }
    WF_DEV bool may_be_visible(int handle) const { return handle == kUnconditional || handle == 0; }
    WF_DEV void term(V3 c, int handle) {
        if (may_be_visible(handle)) radiance += c;
    }
    WF_DEV void kill_if_visible(int handle) {
        if (handle == 0) killed = true;
    }
    WF_DEV void apply_kill(Path& path) const {
        if (killed) path.active = false;
    }
};

struct DeferredSink {
    static constexpr bool kDeferredGather = true;  // caustic gathers go to GatherQueue
    GatherQueue gathers;
    // shadow queue
    float4* shadow_origin;   // origin xyz, t_max
    float4* shadow_dir;      // direction xyz, owner bits
    uint32_t* shadow_count;
    uint32_t shadow_capacity;
    // terms of this path (queue position)
    float4* terms;           // kMaxTerms per queue entry: rgb, handle bits
    uint32_t owner;
    uint32_t tag;            // stored with each shadow request (the batch's job index)
    int nterms;
    int kill;
    uint32_t* overflow;
    WF_DEV int request(V3 o, V3 d, float t_max) {
        unsigned mask = __activemask();
        int lane = threadIdx.x & 31;
        int leader = __ffs(mask) - 1;
        uint32_t base = 0;
        if (lane == leader) base = atomicAdd(shadow_count, uint32_t(__popc(mask)));
        base = __shfl_sync(mask, base, leader);
        uint32_t slot = base + __popc(mask & ((1u << lane) - 1u));
        if (slot >= shadow_capacity) {
            atomicOr(overflow, 1u);
            return kUnconditional;
        }
        shadow_origin[slot] = make_float4(o.x, o.y, o.z, t_max);
        shadow_dir[slot] = make_float4(d.x, d.y, d.z, __uint_as_float(tag));
        return int(slot);
    }
    WF_DEV bool may_be_visible(int) const { return true; }
    WF_DEV void term(V3 c, int handle) {
        if (nterms < kMaxTerms) terms[nterms] = make_float4(c.x, c.y, c.z, __int_as_float(handle));
        ++nterms;
    }
    WF_DEV void kill_if_visible(int handle) { kill = handle; }
    WF_DEV void apply_kill(Path&) const {}
    // Reserves this path's next term for a caustic gather and queues it.
    WF_DEV void gather(const Path& path, const ShadeHit& shaded, V3 albedo) {
        int k = nterms;
        term(V3{0.0f, 0.0f, 0.0f}, kUnconditional);
        if (k >= kMaxTerms) return;  // overflow is reported by the caller
        unsigned mask = __activemask();
        int lane = threadIdx.x & 31;
        int leader = __ffs(mask) - 1;
        uint32_t base = 0;
        if (lane == leader) base = atomicAdd(gathers.count, uint32_t(__popc(mask)));
        base = __shfl_sync(mask, base, leader);
        uint32_t slot = base + __popc(mask & ((1u << lane) - 1u));
        if (slot >= gathers.capacity) {
            atomicOr(overflow, 4u);
            return;
        }
        uint32_t index = owner * kMaxTerms + uint32_t(k);
        gathers.position[slot] = make_float4(shaded.position.x, shaded.position.y, shaded.position.z,
                                             __uint_as_float(index));
        gathers.normal[slot] = make_float4(shaded.normal.x, shaded.normal.y, shaded.normal.z,
                                           path.depth > 0 ? 1.0f : 0.0f);
        gathers.throughput[slot] = make_float4(path.throughput.x, path.throughput.y, path.throughput.z, 0.0f);
        gathers.albedo[slot] = make_float4(albedo.x, albedo.y, albedo.z, 0.0f);
    }
};

// ------------------------------------------------------- next events
// sampleDirectLight, device_traversal.cuh:529-569.
template <typename Sink>
WF_DEV void sample_direct_light(const DeviceScene& s, const RenderParams& rp, Path& path, const ShadeHit& hit,
                                const ShadeHit& shaded, const Material& m, Sink& sink) {
    if (s.light_count == 0) return;
    uint32_t strategy = rp.rng;
    uint32_t candidate = min(uint32_t(random_float(path.rng, strategy) * s.light_count), s.light_count - 1);
    const Light* cl = &s.lights[candidate];
    uint32_t li = random_float(path.rng, strategy) < cl->alias_probability ? candidate : cl->alias;
    const Light& light = s.lights[li];
    float root_u = sqrtf(random_float(path.rng, strategy));
    float v = random_float(path.rng, strategy);
    V3 light_position = (1.0f - root_u) * light.v0 + root_u * (1.0f - v) * light.v1 + root_u * v * light.v2;
    V3 to_light = light_position - hit.position;
    float distance_squared = length_squared(to_light);
    float distance = sqrtf(distance_squared);
    V3 direction = to_light / distance;
    float geometric_cosine = fmaxf(0.0f, dot(hit.geometric_normal, direction));
    float shading_cosine = fmaxf(0.0f, dot(shaded.normal, direction));
    float light_cosine = fmaxf(0.0f, dot(light.normal, -direction));
    bool gltf = (m.flags & kMatGltfPbr) != 0;
    if (geometric_cosine == 0.0f || (!gltf && shading_cosine == 0.0f) || light_cosine == 0.0f) return;
    V3 shadow_origin = offset_ray_origin(hit.position, hit.geometric_normal, direction, hit.t);
    V3 shadow_target = offset_ray_origin(light_position, light.normal, -direction, distance);
    V3 segment = shadow_target - shadow_origin;
    float shadow_distance = length(segment);
    if (!(shadow_distance > kRayMinDistance)) return;
    int handle = kUnconditional;
    if (!s.ignore_direct_light_occlusion)
        handle = sink.request(shadow_origin, segment / shadow_distance, shadow_distance - kRayMinDistance);
    if (!sink.may_be_visible(handle)) return;
    const Material& lm = s.materials[light.material];
    float geometry_term = light_cosine * light.area / (distance_squared * light.selection_pdf);
    float light_pdf = light.selection_pdf * distance_squared / (light_cosine * light.area);
    float bsdf_pdf;
    V3 bsdf = evaluate_surface_cos(s, m, hit, shaded, -path.direction, direction, bsdf_pdf);
    float mis = power_heuristic(light_pdf, bsdf_pdf);
    V3 direct = hadamard(bsdf, lm.emission) * (geometry_term * mis);
    sink.term(clamp_contribution(path, hadamard(path.throughput, direct), rp.clamp, false), handle);
}

// samplePunctualLight, include/scene/punctual_light.cuh:24-50.
struct PunctualSample {
    V3 direction, incident;
    float distance;
};
WF_DEV PunctualSample sample_punctual(const Punctual& light, V3 point) {
    PunctualSample r;
    r.direction = V3{0, 0, 0};
    r.incident = V3{0, 0, 0};
    r.distance = 1.0e30f;
    if (light.type == 2u) {
        r.direction = -light.direction;
        r.incident = light.intensity;
        return r;
    }
    V3 offset = light.position - point;
    float dsq = length_squared(offset);
    if (!(dsq > 0.0f)) return r;
    r.distance = sqrtf(dsq);
    r.direction = offset / r.distance;
    float attenuation = 1.0f / dsq;
    if (light.range > 0.0f) {
        float ratio = r.distance / light.range;
        attenuation *= fmaxf(0.0f, 1.0f - ratio * ratio * ratio * ratio);
    }
    if (light.type == 1u) {
        float cosine = dot(light.direction, -r.direction);
        float cone = fminf(1.0f, fmaxf(0.0f, (cosine - light.outer_cone_cos) /
                                                   fmaxf(1.0e-6f, light.inner_cone_cos - light.outer_cone_cos)));
        attenuation *= cone * cone;
    }
    r.incident = light.intensity * attenuation;
    return r;
}

// addPunctualLight, device_traversal.cuh:653-674.
template <typename Sink>
WF_DEV void add_punctual_light(const DeviceScene& s, const RenderParams& rp, Path& path, const ShadeHit& hit,
                               const ShadeHit& shaded, const Material& m, const Punctual& source,
                               float inverse_selection_pdf, Sink& sink) {
    PunctualSample light = sample_punctual(source, hit.position);
    float cosine = dot(shaded.normal, light.direction);
    bool gltf = (m.flags & kMatGltfPbr) != 0;
    if ((!gltf && cosine <= 0.0f) || dot(hit.geometric_normal, light.direction) <= 0.0f ||
        length_squared(light.incident) == 0.0f)
        return;
    V3 origin = offset_ray_origin(hit.position, hit.geometric_normal, light.direction, hit.t);
    V3 direction = light.direction;
    float shadow_distance = light.distance;
    if (source.type != 2u) {
        V3 segment = source.position - origin;
        shadow_distance = length(segment);
        if (!(shadow_distance > kRayMinDistance)) return;
        direction = segment / shadow_distance;
    }
    int handle = kUnconditional;
    if (!s.ignore_direct_light_occlusion) handle = sink.request(origin, direction, shadow_distance - kRayMinDistance);
    if (!sink.may_be_visible(handle)) return;
    float ignored;
    V3 bsdf = evaluate_surface_cos(s, m, hit, shaded, -path.direction, light.direction, ignored);
    V3 direct = hadamard(bsdf, light.incident) * inverse_selection_pdf;
    sink.term(clamp_contribution(path, hadamard(path.throughput, direct), rp.clamp, false), handle);
}

// sampleDirectPunctualLight, device_traversal.cuh:676-683.
template <typename Sink>
WF_DEV void sample_direct_punctual(const DeviceScene& s, const RenderParams& rp, Path& path, const ShadeHit& hit,
                                   const ShadeHit& shaded, const Material& m, Sink& sink) {
    for (uint32_t i = 0; i < s.directional_count; ++i)
        add_punctual_light(s, rp, path, hit, shaded, m, s.punctual[i], 1.0f, sink);
    uint32_t count = s.punctual_count - s.directional_count;
    if (count == 0) return;
    uint32_t index = s.directional_count + min(uint32_t(random_float(path.rng, rp.rng) * count), count - 1);
    add_punctual_light(s, rp, path, hit, shaded, m, s.punctual[index], float(count), sink);
}

// sampleDirectEnvironment, device_traversal.cuh:637-651.
template <typename Sink>
WF_DEV void sample_direct_environment(const DeviceScene& s, const RenderParams& rp, Path& path, const ShadeHit& hit,
                                      const ShadeHit& shaded, const Material& m, Sink& sink) {
    const Environment& e = s.env;
    if (!e.present || e.intensity == 0.0f) return;
    EnvSample light = sample_path_environment(s, path, rp.rng);
    float cosine = dot(shaded.normal, light.direction);
    bool gltf = (m.flags & kMatGltfPbr) != 0;
    if ((!gltf && cosine <= 0.0f) || dot(hit.geometric_normal, light.direction) <= 0.0f || !(light.pdf > 0.0f)) return;
    V3 origin = offset_ray_origin(hit.position, hit.geometric_normal, light.direction, hit.t);
    int handle = kUnconditional;
    if (!s.ignore_direct_light_occlusion) handle = sink.request(origin, light.direction, 1.0e30f);
    if (!sink.may_be_visible(handle)) return;
    float bsdf_pdf;
    V3 bsdf = evaluate_surface_cos(s, m, hit, shaded, -path.direction, light.direction, bsdf_pdf);
    float weight = power_heuristic(light.pdf, bsdf_pdf);
    V3 direct = hadamard(bsdf, environment_radiance(e, light.direction)) * (weight / light.pdf);
    sink.term(clamp_contribution(path, hadamard(path.throughput, direct), rp.clamp, false), handle);
}

// addEnvironmentOrSky, device_traversal.cuh:577-587.
template <typename Sink>
WF_DEV void add_environment_or_sky(const DeviceScene& s, const RenderParams& rp, const Path& path, Sink& sink) {
    if (s.env.present) {
        float weight = path.depth > 0 && !path.specular
                           ? power_heuristic(path.prev_pdf, environment_pdf(s.env, path.direction))
                           : 1.0f;
        V3 c = hadamard(path.throughput, environment_radiance(s.env, path.direction)) * weight;
        sink.term(clamp_contribution(path, c, rp.clamp, true), kUnconditional);
    } else if (!s.black_background) {
        float t = 0.5f * (path.direction.y + 1.0f);
        V3 sky = (1.0f - t) * V3{1.0f, 1.0f, 1.0f} + t * V3{0.5f, 0.7f, 1.0f};
        sink.term(clamp_contribution(path, hadamard(path.throughput, sky), rp.clamp, true), kUnconditional);
    }
}

// ------------------------------------------------------------ caustics
// gatherCaustics, src/renderer/photon_mapping.cu:91-163, over a grid whose
// cells list their photons in the order the reference's serial insertion
// produces (descending photon index).
WF_DEV V3 gather_caustics(const PhotonGridView& g, const ShadeHit& hit, float radius) {
    // Every stored photon lies inside [minimum, maximum] (the grid drops the
    // others), so a point farther than the search radius from that box finds
    // no candidate: the reference then returns zero (nearestCount == 0) after
    // scanning the clamped border cells.  Return it directly.
    {
        float sr = fmaxf(radius * 4.0f, 0.1f) * 1.001f;  // margin keeps the test strict after rounding
        float dx = fmaxf(fmaxf(g.minimum.x - hit.position.x, hit.position.x - g.maximum.x), 0.0f);
        float dy = fmaxf(fmaxf(g.minimum.y - hit.position.y, hit.position.y - g.maximum.y), 0.0f);
        float dz = fmaxf(fmaxf(g.minimum.z - hit.position.z, hit.position.z - g.maximum.z), 0.0f);
        if (dx > sr || dy > sr || dz > sr) return V3{0, 0, 0};
    }
    V3 extent = g.maximum - g.minimum;
    V3 offset = hit.position - g.minimum;
    V3 nrm{offset.x / extent.x, offset.y / extent.y, offset.z / extent.z};
    int res = int(g.resolution);
    int cx = min(max(int(nrm.x * g.resolution), 0), res - 1);
    int cy = min(max(int(nrm.y * g.resolution), 0), res - 1);
    int cz = min(max(int(nrm.z * g.resolution), 0), res - 1);
    constexpr uint32_t kMaxNearest = 64;
    constexpr uint32_t kMinimumPhotons = 16;
    float search_radius = fmaxf(radius * 4.0f, 0.1f);
    int cell_radius = max(1, int(ceilf(search_radius * g.resolution / fmaxf(extent.x, 0.0001f))));
    float search_sq = search_radius * search_radius;
    float nearest_d[kMaxNearest];
    uint32_t nearest_i[kMaxNearest];
    uint32_t count = 0, farthest = 0;
    float farthest_sq = 0.0f;
    for (uint32_t i = 0; i < kMaxNearest; ++i) {
        nearest_d[i] = 0.0f;
        nearest_i[i] = kInvalid;
    }
    for (int z = cz - cell_radius; z <= cz + cell_radius; ++z)
        for (int y = cy - cell_radius; y <= cy + cell_radius; ++y)
            for (int x = cx - cell_radius; x <= cx + cell_radius; ++x) {
                if (x < 0 || y < 0 || z < 0 || x >= res || y >= res || z >= res) continue;
                // A cell whose box (padded by a rounding margin) lies beyond the
                // search radius holds no photon the distance test accepts, so
                // skipping it leaves the accepted sequence unchanged.
                {
                    float cx0 = g.minimum.x + extent.x * (float(x) / float(res));
                    float cx1 = g.minimum.x + extent.x * (float(x + 1) / float(res));
                    float cy0 = g.minimum.y + extent.y * (float(y) / float(res));
                    float cy1 = g.minimum.y + extent.y * (float(y + 1) / float(res));
                    float cz0 = g.minimum.z + extent.z * (float(z) / float(res));
                    float cz1 = g.minimum.z + extent.z * (float(z + 1) / float(res));
                    float gx = fmaxf(fmaxf(cx0 - hit.position.x, hit.position.x - cx1), 0.0f);
                    float gy = fmaxf(fmaxf(cy0 - hit.position.y, hit.position.y - cy1), 0.0f);
                    float gz = fmaxf(fmaxf(cz0 - hit.position.z, hit.position.z - cz1), 0.0f);
                    float cell_margin = search_radius * 1.001f + 1.0e-4f * (fabsf(extent.x) + fabsf(extent.y) + fabsf(extent.z));
                    if (gx > cell_margin || gy > cell_margin || gz > cell_margin) continue;
                }
                uint32_t cell = (uint32_t(z) * g.resolution + uint32_t(y)) * g.resolution + uint32_t(x);
                uint32_t begin = g.cell_start[cell], end = begin + g.cell_count[cell];
                for (uint32_t p = begin; p < end; ++p) {
                    float4 pp = __ldg(&g.position[p]);
                    V3 po = V3{pp.x, pp.y, pp.z} - hit.position;
                    float dsq = dot(po, po);
                    if (dsq > search_sq) continue;  // the direction is read only for photons in range
                    float4 pd = __ldg(&g.direction[p]);
                    float cosine = dot(hit.normal, V3{pd.x, pd.y, pd.z});
                    if (cosine <= 0.0f) continue;
                    if (count < kMaxNearest) {
                        nearest_d[count] = dsq;
                        nearest_i[count] = p;
                        if (dsq > farthest_sq) {
                            farthest_sq = dsq;
                            farthest = count;
                        }
                        ++count;
                    } else if (dsq < farthest_sq) {
                        nearest_d[farthest] = dsq;
                        nearest_i[farthest] = p;
                        farthest = 0;
                        farthest_sq = nearest_d[0];
                        for (uint32_t i = 1; i < kMaxNearest; ++i)
                            if (nearest_d[i] > farthest_sq) {
                                farthest_sq = nearest_d[i];
                                farthest = i;
                            }
                    }
                }
            }
    if (count == 0) return V3{0, 0, 0};
    float gather_sq = search_sq;
    if (count >= kMinimumPhotons) {
        gather_sq = 0.0f;
        for (uint32_t i = 0; i < count; ++i) gather_sq = fmaxf(gather_sq, nearest_d[i]);
        gather_sq = fmaxf(gather_sq, radius * radius);
    }
    float gather_radius = sqrtf(gather_sq);
    V3 result{0, 0, 0};
    for (uint32_t i = 0; i < count; ++i) {
        float4 pd = __ldg(&g.direction[nearest_i[i]]);
        float4 pf = __ldg(&g.flux[nearest_i[i]]);
        float distance = sqrtf(nearest_d[i]);
        float cone = fmaxf(0.0f, 1.0f - distance / gather_radius);
        result += V3{pf.x, pf.y, pf.z} * (cone * dot(hit.normal, V3{pd.x, pd.y, pd.z}));
    }
    return result * (3.0f / (3.14159265359f * gather_sq));
}

// Photons stored in the cells gather_caustics scans for this point (an upper
// bound on its candidates: the cost of the serial scan).
WF_DEV uint32_t gather_cell_photons(const PhotonGridView& g, V3 position, float radius) {
    {
        float sr = fmaxf(radius * 4.0f, 0.1f) * 1.001f;
        float dx = fmaxf(fmaxf(g.minimum.x - position.x, position.x - g.maximum.x), 0.0f);
        float dy = fmaxf(fmaxf(g.minimum.y - position.y, position.y - g.maximum.y), 0.0f);
        float dz = fmaxf(fmaxf(g.minimum.z - position.z, position.z - g.maximum.z), 0.0f);
        if (dx > sr || dy > sr || dz > sr) return 0;
    }
    V3 extent = g.maximum - g.minimum;
    V3 offset = position - g.minimum;
    V3 nrm{offset.x / extent.x, offset.y / extent.y, offset.z / extent.z};
    int res = int(g.resolution);
    int cx = min(max(int(nrm.x * g.resolution), 0), res - 1);
    int cy = min(max(int(nrm.y * g.resolution), 0), res - 1);
    int cz = min(max(int(nrm.z * g.resolution), 0), res - 1);
    float search_radius = fmaxf(radius * 4.0f, 0.1f);
    int cell_radius = max(1, int(ceilf(search_radius * g.resolution / fmaxf(extent.x, 0.0001f))));
    uint32_t total = 0;
    for (int z = max(cz - cell_radius, 0); z <= min(cz + cell_radius, res - 1); ++z)
        for (int y = max(cy - cell_radius, 0); y <= min(cy + cell_radius, res - 1); ++y)
            for (int x = max(cx - cell_radius, 0); x <= min(cx + cell_radius, res - 1); ++x)
                total += g.cell_count[(uint32_t(z) * g.resolution + uint32_t(y)) * g.resolution + uint32_t(x)];
    return total;
}

// gather_caustics for one shading point, computed by a whole warp (all 32
// lanes call it with the same arguments).  The lanes filter 32 photons of a
// cell at a time; the photons that pass are then inserted one after another
// in scan order, exactly as the serial loop does, into the 64-entry nearest
// set, whose entries i and i + 32 live in lane i.  The farthest entry (the
// first index holding the largest distance) is found by a warp argmax, and
// the result is summed serially in slot order, so the value is the serial
// one bit for bit.  Every lane returns the result.
WF_DEV V3 gather_caustics_warp(const PhotonGridView& g, V3 position, V3 normal, float radius) {
    const uint32_t lane = threadIdx.x & 31;
    {
        float sr = fmaxf(radius * 4.0f, 0.1f) * 1.001f;
        float dx = fmaxf(fmaxf(g.minimum.x - position.x, position.x - g.maximum.x), 0.0f);
        float dy = fmaxf(fmaxf(g.minimum.y - position.y, position.y - g.maximum.y), 0.0f);
        float dz = fmaxf(fmaxf(g.minimum.z - position.z, position.z - g.maximum.z), 0.0f);
        if (dx > sr || dy > sr || dz > sr) return V3{0, 0, 0};
    }
    V3 extent = g.maximum - g.minimum;
    V3 offset = position - g.minimum;
    V3 nrm{offset.x / extent.x, offset.y / extent.y, offset.z / extent.z};
    int res = int(g.resolution);
    int cx = min(max(int(nrm.x * g.resolution), 0), res - 1);
    int cy = min(max(int(nrm.y * g.resolution), 0), res - 1);
    int cz = min(max(int(nrm.z * g.resolution), 0), res - 1);
    constexpr uint32_t kMaxNearest = 64;
    constexpr uint32_t kMinimumPhotons = 16;
    float search_radius = fmaxf(radius * 4.0f, 0.1f);
    int cell_radius = max(1, int(ceilf(search_radius * g.resolution / fmaxf(extent.x, 0.0001f))));
    float search_sq = search_radius * search_radius;
    // entries lane and lane + 32 of the nearest set
    float near_d[2] = {0.0f, 0.0f};
    uint32_t near_i[2] = {kInvalid, kInvalid};
    uint32_t count = 0, farthest = 0;
    float farthest_sq = 0.0f;
    for (int z = cz - cell_radius; z <= cz + cell_radius; ++z)
        for (int y = cy - cell_radius; y <= cy + cell_radius; ++y)
            for (int x = cx - cell_radius; x <= cx + cell_radius; ++x) {
                if (x < 0 || y < 0 || z < 0 || x >= res || y >= res || z >= res) continue;
                {
                    float cx0 = g.minimum.x + extent.x * (float(x) / float(res));
                    float cx1 = g.minimum.x + extent.x * (float(x + 1) / float(res));
                    float cy0 = g.minimum.y + extent.y * (float(y) / float(res));
                    float cy1 = g.minimum.y + extent.y * (float(y + 1) / float(res));
                    float cz0 = g.minimum.z + extent.z * (float(z) / float(res));
                    float cz1 = g.minimum.z + extent.z * (float(z + 1) / float(res));
                    float gx = fmaxf(fmaxf(cx0 - position.x, position.x - cx1), 0.0f);
                    float gy = fmaxf(fmaxf(cy0 - position.y, position.y - cy1), 0.0f);
                    float gz = fmaxf(fmaxf(cz0 - position.z, position.z - cz1), 0.0f);
                    float cell_margin = search_radius * 1.001f + 1.0e-4f * (fabsf(extent.x) + fabsf(extent.y) + fabsf(extent.z));
                    if (gx > cell_margin || gy > cell_margin || gz > cell_margin) continue;
                }
                uint32_t cell = (uint32_t(z) * g.resolution + uint32_t(y)) * g.resolution + uint32_t(x);
                uint32_t begin = g.cell_start[cell], end = begin + g.cell_count[cell];
                for (uint32_t base = begin; base < end; base += 32) {
                    uint32_t p = base + lane;
                    float dsq = 0.0f;
                    bool accept = false;
                    if (p < end) {
                        float4 pp = __ldg(&g.position[p]);
                        V3 po = V3{pp.x, pp.y, pp.z} - position;
                        dsq = dot(po, po);
                        if (!(dsq > search_sq)) {  // the serial loop's rejection tests, negated
                            float4 pd = __ldg(&g.direction[p]);
                            accept = !(dot(normal, V3{pd.x, pd.y, pd.z}) <= 0.0f);
                        }
                    }
                    unsigned accepted = __ballot_sync(0xffffffffu, accept);
                    while (accepted) {
                        int j = __ffs(accepted) - 1;
                        accepted &= accepted - 1;
                        float d = __shfl_sync(0xffffffffu, dsq, j);
                        uint32_t index = base + uint32_t(j);
                        if (count < kMaxNearest) {
                            if ((count & 31) == lane) {
                                near_d[count >> 5] = d;
                                near_i[count >> 5] = index;
                            }
                            if (d > farthest_sq) {
                                farthest_sq = d;
                                farthest = count;
                            }
                            ++count;
                        } else if (d < farthest_sq) {
                            if ((farthest & 31) == lane) {
                                near_d[farthest >> 5] = d;
                                near_i[farthest >> 5] = index;
                            }
                            // first index holding the largest distance
                            float best = near_d[1] > near_d[0] ? near_d[1] : near_d[0];
                            uint32_t at = near_d[1] > near_d[0] ? lane + 32 : lane;
                            for (int off = 16; off > 0; off >>= 1) {
                                float ob = __shfl_xor_sync(0xffffffffu, best, off);
                                uint32_t oa = __shfl_xor_sync(0xffffffffu, at, off);
                                if (ob > best || (ob == best && oa < at)) {
                                    best = ob;
                                    at = oa;
                                }
                            }
                            farthest_sq = best;
                            farthest = at;
                        }
                    }
                }
            }
    if (count == 0) return V3{0, 0, 0};
    float gather_sq = search_sq;
    if (count >= kMinimumPhotons) {
        float m = 0.0f;
        if (lane < count) m = fmaxf(m, near_d[0]);
        if (lane + 32 < count) m = fmaxf(m, near_d[1]);
        for (int off = 16; off > 0; off >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, off));
        gather_sq = fmaxf(m, radius * radius);
    }
    float gather_radius = sqrtf(gather_sq);
    V3 part[2];
    for (int h = 0; h < 2; ++h) {
        part[h] = V3{0.0f, 0.0f, 0.0f};
        if (lane + 32u * h < count) {
            float4 pd = __ldg(&g.direction[near_i[h]]);
            float4 pf = __ldg(&g.flux[near_i[h]]);
            float distance = sqrtf(near_d[h]);
            float cone = fmaxf(0.0f, 1.0f - distance / gather_radius);
            part[h] = V3{pf.x, pf.y, pf.z} * (cone * dot(normal, V3{pd.x, pd.y, pd.z}));
        }
    }
    V3 result{0, 0, 0};
    for (uint32_t i = 0; i < count; ++i) {  // slot order, as the serial sum
        int src = int(i & 31);
        V3 c = (i >> 5) ? part[1] : part[0];
        result.x += __shfl_sync(0xffffffffu, c.x, src);
        result.y += __shfl_sync(0xffffffffu, c.y, src);
        result.z += __shfl_sync(0xffffffffu, c.z, src);
    }
    return result * (3.0f / (3.14159265359f * gather_sq));
}

// --------------------------------------------------------- continuations
// continueDielectricSurface, device_traversal.cuh:589-635.
template <typename Sink>
WF_DEV V3 continue_dielectric(const DeviceScene& s, const RenderParams& rp, Path& path, const ShadeHit& hit,
                              const ShadeHit& shaded, const Material& m, Sink& sink) {
    path.throughput = hadamard(path.throughput, m.albedo);
    DielectricInterface b = dielectric_interface(normalize(path.direction), hit.geometric_normal, shaded.normal, m.ior);
    float eta_sq = b.eta * b.eta;
    int reflection_test = kUnconditional, transmission_test = kUnconditional;
    if (s.env.present && path.depth + 1 < rp.max_depth) {
        if (b.reflectance > 0.0f) {
            V3 d = b.reflection;
            reflection_test = sink.request(offset_ray_origin(hit.position, hit.geometric_normal, d, hit.t), d, 1.0e30f);
            if (sink.may_be_visible(reflection_test)) {
                V3 c = hadamard(path.throughput, environment_radiance(s.env, d)) * b.reflectance;
                sink.term(clamp_contribution(path, c, rp.clamp, false), reflection_test);
            }
        }
        if (b.reflectance < 1.0f) {
            V3 d = b.transmission;
            transmission_test = sink.request(offset_ray_origin(hit.position, hit.geometric_normal, d, hit.t), d, 1.0e30f);
            if (sink.may_be_visible(transmission_test)) {
                V3 c = hadamard(path.throughput, environment_radiance(s.env, d)) * ((1.0f - b.reflectance) * eta_sq);
                sink.term(clamp_contribution(path, c, rp.clamp, false), transmission_test);
            }
        }
    }
    bool reflected = b.reflectance >= 1.0f || b.reflectance > random_float(path.rng, rp.rng);
    if (!reflected) {
        path.throughput *= eta_sq;
        path.eta_scale /= eta_sq;
        if (b.front_face) {
            path.medium = hit.material;
            path.medium_density = m.volume_density * 1.0f;
        } else {
            path.medium = kInvalid;
            path.medium_density = 1.0f;
        }
    }
    int escape = reflected ? reflection_test : transmission_test;
    if (escape != kUnconditional) sink.kill_if_visible(escape);
    path.specular = true;
    path.prev_pdf = 0.0f;
    return reflected ? b.reflection : b.transmission;
}

// continueDiffuseSurface, device_traversal.cuh:685-704.
WF_DEV V3 continue_diffuse(const DeviceScene& s, const RenderParams& rp, Path& path, const ShadeHit& hit,
                           const ShadeHit& shaded, const Material& m) {
    float probability = s.env.sampling ? 0.5f : 0.0f;
    V3 direction = probability > 0.0f && random_float(path.rng, rp.rng) < probability
                       ? sample_path_environment(s, path, rp.rng).direction
                       : sample_cosine_hemisphere(shaded.normal, path, rp.rng);
    float cosine = dot(shaded.normal, direction);
    float pdf = diffuse_continuation_pdf(s, shaded.normal, direction);
    if (!(pdf > 0.0f) || cosine <= 0.0f || dot(direction, hit.geometric_normal) <= 0.0f) {
        path.active = false;
        return direction;
    }
    path.throughput = hadamard(path.throughput, m.albedo) * (cosine * 0.31830988618f / pdf);
    path.prev_pdf = pdf;
    path.specular = false;
    return direction;
}

// continueGlossySurface, device_traversal.cuh:706-725.
WF_DEV V3 continue_glossy(const DeviceScene& s, const RenderParams& rp, Path& path, const ShadeHit& hit,
                          const ShadeHit& shaded, const Material& m) {
    SpecGloss surface = m.type == kSpecGloss ? SpecGloss{m.albedo, m.specular, material_roughness(m)}
                                             : SpecGloss{V3{0, 0, 0}, m.albedo, material_roughness(m)};
    V3 outgoing = -path.direction;
    float choice = random_float(path.rng, rp.rng);
    float u = random_float(path.rng, rp.rng);
    float v = random_float(path.rng, rp.rng);
    V3 direction = sg_sample(surface, shaded.normal, outgoing, choice, u, v);
    float pdf;
    V3 bsdf = sg_evaluate(surface, shaded.normal, outgoing, direction, pdf);
    if (!(pdf > 0.0f) || dot(direction, hit.geometric_normal) <= 0.0f) {
        path.active = false;
        return direction;
    }
    path.throughput = hadamard(path.throughput, bsdf) * (fmaxf(0.0f, dot(shaded.normal, direction)) / pdf);
    path.prev_pdf = pdf;
    path.specular = false;
    return direction;
}

// continueGltfPbrSurface, device_traversal.cuh:727-787.
template <typename Sink>
WF_DEV V3 continue_gltf(const DeviceScene& s, const RenderParams& rp, Path& path, const ShadeHit& hit,
                        const ShadeHit& shaded, const Material& m, Sink& sink) {
    GltfPbr g = gltf_surface(m, hit, shaded);
    V3 view = -path.direction;
    correct_gltf_normals(g, hit.geometric_normal, view);
    GltfWeights w = pbr_weights(g, view);
    float choice = random_float(path.rng, rp.rng);
    bool coat = choice < w.coat;
    bool specular = !coat && choice < w.coat + w.specular;
    bool delta = (coat && g.coat_roughness <= 0) || (specular && g.roughness <= 0);
    int base_test = kUnconditional, coat_test = kUnconditional;
    V3 base_coefficient = pbr_base_fresnel(g, dot(pbr_specular_normal(g), view)) * (1.f - w.coat);
    if (s.env.present && path.depth + 1 < rp.max_depth) {
        for (int lobe = 0; lobe < 2; ++lobe) {
            bool is_coat = lobe == 1;
            float mass = is_coat ? w.coat : w.specular;
            float roughness = is_coat ? g.coat_roughness : g.roughness;
            if (!(mass > 0) || roughness > 0) continue;
            V3 normal = is_coat ? g.coat_normal : pbr_specular_normal(g);
            V3 direction = pbr_sample_reflection(normal, view, 0, 0, 0);
            if (dot(normal, view) <= 0 || dot(direction, hit.geometric_normal) <= 0) continue;
            int test = sink.request(offset_ray_origin(hit.position, hit.geometric_normal, direction, hit.t), direction,
                                    1.e30f);
            if (is_coat) coat_test = test; else base_test = test;
            if (sink.may_be_visible(test)) {
                V3 coefficient = is_coat ? V3{w.coat, w.coat, w.coat} : base_coefficient;
                V3 c = hadamard(path.throughput, hadamard(coefficient, environment_radiance(s.env, direction)));
                sink.term(clamp_contribution(path, c, rp.clamp, false), test);
            }
        }
    }
    V3 direction;
    if (coat || specular) {
        float u = random_float(path.rng, rp.rng);
        float v = random_float(path.rng, rp.rng);
        V3 normal = coat ? g.coat_normal : pbr_specular_normal(g);
        direction = pbr_sample_reflection(normal, view, coat ? g.coat_roughness : g.roughness, u, v);
        if (dot(normal, view) <= 0) {
            path.active = false;
            return direction;
        }
    } else {
        float probability = s.env.sampling ? 0.5f : 0.0f;
        direction = probability > 0 && random_float(path.rng, rp.rng) < probability
                        ? sample_path_environment(s, path, rp.rng).direction
                        : sample_cosine_hemisphere(g.normal, path, rp.rng);
    }
    if (dot(direction, hit.geometric_normal) <= 0) {
        path.active = false;
        return direction;
    }
    if (delta) {
        float mass = coat ? w.coat : w.specular;
        V3 coefficient = coat ? V3{w.coat, w.coat, w.coat} : base_coefficient;
        path.throughput = hadamard(path.throughput, coefficient) / mass;
        path.specular = true;
        path.prev_pdf = 0;
        int escape = coat ? coat_test : base_test;
        if (escape != kUnconditional) sink.kill_if_visible(escape);
    } else {
        float pdf;
        V3 value = pbr_evaluate_cos(g, view, direction, diffuse_continuation_pdf(s, g.normal, direction), pdf);
        if (!(pdf > 0)) {
            path.active = false;
            return direction;
        }
        path.throughput = hadamard(path.throughput, value) / pdf;
        path.prev_pdf = pdf;
        path.specular = false;
    }
    return direction;
}

// --------------------------------------------------------------- shade
// shadePaths / shadePersistentPath, device_path_shading.cuh:6-173,175-319.
// Returns false when the path ends with this event (the caller then adds the
// path radiance to the framebuffer); the sink may still end it through a
// visible terminal branch.
// kTextures = false compiles the texture code out, for kernels the host
// launches only on scenes without textured materials.
template <typename Sink, bool kTextures = true>
WF_DEV bool shade_path(const DeviceScene& s, const RenderParams& rp, Path& path, bool did_hit, const SurfaceHit& sh,
                       Sink& sink) {
    if (rp.debug == 1 || rp.debug == 2) {
        V3 color{0.05f, 0.10f, 0.25f};
        V3 n = sh.normal;
        if constexpr (kTextures) {
            if (did_hit && rp.debug == 2 && (s.materials[sh.material].flags & kMatTextured) && s.material_textures) {
                const MaterialTextures& mt = s.material_textures[sh.material];
                n = material_normal(s, mt.slot[kTexNormal], mt.normal_scale, sh);
            }
        }
        if (did_hit) color = 0.5f * (n + V3{1.0f, 1.0f, 1.0f});
        sink.term(color, kUnconditional);
        path.active = false;
        return false;
    }
    if (!did_hit) {
        add_environment_or_sky(s, rp, path, sink);
        path.active = false;
        return false;
    }
    ShadeHit hit{sh.t, sh.position, sh.geometric_normal, sh.normal, sh.material, sh.light, sh.normal};
    const Material& stored = s.materials[hit.material];
    bool textured = false;
    Material resolved;
    if constexpr (kTextures) {
        textured = (stored.flags & kMatTextured) && s.material_textures;
        if (textured) resolved = resolve_material(s, stored, hit.material, sh);
    }
    const Material& m = textured ? resolved : stored;
    if (path.medium != kInvalid) {
        const Material& medium = s.materials[path.medium];
        if (medium.attenuation_distance > 0.0f) {
            float distance = hit.t * path.medium_density;
            V3 sigma{-wfm::logf(fmaxf(medium.attenuation_color.x, 0.0001f)) / medium.attenuation_distance,
                     -wfm::logf(fmaxf(medium.attenuation_color.y, 0.0001f)) / medium.attenuation_distance,
                     -wfm::logf(fmaxf(medium.attenuation_color.z, 0.0001f)) / medium.attenuation_distance};
            path.throughput = hadamard(path.throughput, V3{wfm::expf(-sigma.x * distance), wfm::expf(-sigma.y * distance),
                                                           wfm::expf(-sigma.z * distance)});
        }
    }
    if (m.type == kEmissive) {
        float mis = 1.0f;
        if (hit.light != kInvalid) {
            const Light& light = s.lights[hit.light];
            float light_cosine = fmaxf(0.0f, dot(light.normal, -path.direction));
            if (light_cosine == 0.0f)
                mis = 0.0f;
            else if (path.depth > 0 && !path.specular) {
                float light_pdf = light.selection_pdf * hit.t * hit.t / (light_cosine * light.area);
                mis = power_heuristic(path.prev_pdf, light_pdf);
            }
        }
        sink.term(clamp_contribution(path, hadamard(path.throughput, m.emission) * mis, rp.clamp, true),
                  kUnconditional);
        path.active = false;
        return false;
    }
    ShadeHit shaded = hit;
    if (textured) {
        const MaterialTextures& mt = s.material_textures[hit.material];
        shaded.normal = material_normal(s, mt.slot[kTexNormal], mt.normal_scale, sh);
        shaded.coat_normal = material_normal(s, mt.slot[kTexClearcoatNormal], mt.clearcoat_normal_scale, sh);
    }
    if (dot(shaded.normal, hit.geometric_normal) < 0.0f) shaded.normal = -shaded.normal;
    V3 albedo = m.albedo;
    uint32_t type = m.type == kDiffuse && m.metallic > 0.5f ? uint32_t(kMetal) : m.type;
    float roughness = material_roughness(m);
    V3 direction{0, 0, 0};
    // Every non-delta surface samples the triangle lights, the punctual lights
    // and the environment before its continuation (the same order in each
    // material branch of shadePaths); one call site keeps the kernel small.
    bool gltf = (m.flags & kMatGltfPbr) != 0;
    if (gltf || type == kDiffuse || type == kSpecGloss || (type == kMetal && roughness > 0.0f)) {
        sample_direct_light(s, rp, path, hit, shaded, m, sink);
        sample_direct_punctual(s, rp, path, hit, shaded, m, sink);
        sample_direct_environment(s, rp, path, hit, shaded, m, sink);
    }
    if (gltf) {
        direction = continue_gltf(s, rp, path, hit, shaded, m, sink);
    } else if (type == kDiffuse) {
        if (rp.photons.enabled) {
            if constexpr (Sink::kDeferredGather) {
                sink.gather(path, shaded, albedo);
            } else {
                V3 caustic = gather_caustics(rp.photons, shaded, rp.gather_radius);
                sink.term(clamp_contribution(path, hadamard(path.throughput, hadamard(albedo, caustic)), rp.clamp,
                                             false),
                          kUnconditional);
            }
        }
        direction = continue_diffuse(s, rp, path, hit, shaded, m);
    } else if (type == kSpecGloss) {
        direction = continue_glossy(s, rp, path, hit, shaded, m);
    } else if (type == kMetal) {
        if (roughness > 0.0f) {
            direction = continue_glossy(s, rp, path, hit, shaded, m);
        } else {
            path.throughput = hadamard(path.throughput, albedo);
            V3 reflected = reflect(normalize(path.direction), shaded.normal);
            direction = normalize(reflected + roughness * random_in_unit_sphere(path, rp.rng));
            if (dot(direction, shaded.normal) <= 0.0f || dot(direction, hit.geometric_normal) <= 0.0f)
                direction = reflect(normalize(path.direction), hit.geometric_normal);
            path.specular = true;
            path.prev_pdf = 0.0f;
        }
    } else if (type == kDielectric) {
        direction = continue_dielectric(s, rp, path, hit, shaded, m, sink);
    }
    sink.apply_kill(path);
    if (!path.active) return false;
    path.origin = offset_ray_origin(hit.position, hit.geometric_normal, direction, hit.t);
    path.direction = direction;
    ++path.depth;
    if (path.depth >= rp.max_depth) {
        path.active = false;
        return false;
    }
    if (path.depth >= rp.rr_start) {
        float survival = fminf(0.95f, fmaxf(0.05f, path.eta_scale * fmaxf(path.throughput.x,
                                                                          fmaxf(path.throughput.y, path.throughput.z))));
        if (random_float(path.rng, rp.rng) > survival) {
            path.active = false;
            return false;
        }
        path.throughput *= 1.0f / survival;
    }
    return true;
}

// Camera::generateRay, include/scene/camera.cuh:17-27 (tanHalfFov hoisted).
WF_DEV void camera_ray(const Camera& c, float u, float v, V3& origin, V3& direction) {
    float x = (2.0f * u - 1.0f) * c.aspect_ratio * c.tan_half_fov;
    float y = (1.0f - 2.0f * v) * c.tan_half_fov;
    direction = normalize(c.forward + c.right * x + c.up * y);
    origin = c.position;
}

}  // namespace wf
