// ORACLE / TEST INFRASTRUCTURE ONLY -- never linked into or called by the
// product.  Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline
// load the libraries built from this file (oracle/_build/liboracle*.so).
//
// A scalar CPU restatement of the reference renderer's path (one path at a
// time, every bounce in a loop), written from the reference's algorithm:
// RNG keying (include/core/rng.cuh, src/core/rng.cu), camera
// (include/scene/camera.cuh), BVH2/TLAS/BLAS closest hit and any hit
// (include/renderer/device_traversal.cuh), path shading with NEE/MIS over
// triangle lights, punctual lights and the HDR environment, dielectric,
// metal, diffuse continuation and Russian roulette
// (include/renderer/device_path_shading.cuh, device_sampling.cuh,
// specular_glossiness.cuh, environment.cuh), photon caustics
// (src/renderer/photon_mapping.cu), light and environment tables
// (src/scene/scene.cu:82-121, src/scene/environment.cpp:10-64,
// src/scene/scene_host.cpp:60-106).  Not covered here: glTF metal/rough and
// specular-glossiness materials (the host-compiled reference covers those).
//
// Built twice: ORACLE_DET_MATH=0 uses the C library's elementary functions
// (pinned bit for bit against oracle/_ref/libwfref.so), =1 the deterministic
// ones of wf_math.h (pinned against libwfref_det.so).  Trees come from the
// project's BVH builder, as the reference's come from NexusBVH.
#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../include/wavefront.h"
#include "../wavefront-path-tracer_b200/csrc/bvh_build.h"

#if ORACLE_DET_MATH
#include "../wavefront-path-tracer_b200/csrc/wf_math.h"
static float m_sinf(float x) { return wfm::sinf(x); }
static float m_cosf(float x) { return wfm::cosf(x); }
static float m_tanf(float x) { return wfm::tanf(x); }
static float m_atan2f(float y, float x) { return wfm::atan2f(y, x); }
static float m_logf(float x) { return wfm::logf(x); }
static float m_expf(float x) { return wfm::expf(x); }
static float m_powf(float x, float y) { return wfm::powf(x, y); }
static double m_sin(double x) { return wfm::sin(x); }
static double m_cos(double x) { return wfm::cos(x); }
#else
static float m_sinf(float x) { return ::sinf(x); }
static float m_cosf(float x) { return ::cosf(x); }
static float m_tanf(float x) { return ::tanf(x); }
static float m_atan2f(float y, float x) { return ::atan2f(y, x); }
static float m_logf(float x) { return ::logf(x); }
static float m_expf(float x) { return ::expf(x); }
static float m_powf(float x, float y) { return ::powf(x, y); }
static double m_sin(double x) { return ::sin(x); }
static double m_cos(double x) { return ::cos(x); }
#endif

namespace port {

constexpr uint32_t NONE = 0xffffffffu;
constexpr float T_MIN = 1.0e-6f;

// ---------------------------------------------------------------- vectors
struct V {
    float x = 0, y = 0, z = 0;
};
static V mk(float x, float y, float z) { V v; v.x = x; v.y = y; v.z = z; return v; }
static V mk3(const float* p) { return mk(p[0], p[1], p[2]); }
static V add(V a, V b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static V sub(V a, V b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static V neg(V a) { return mk(-a.x, -a.y, -a.z); }
static V mul(V a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
static V divs(V a, float s) { float r = 1.0f / s; return mul(a, r); }
static V had(V a, V b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
static float dot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static V cross(V a, V b) { return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static float len2(V a) { return dot(a, a); }
static float len(V a) { return std::sqrt(len2(a)); }
static V unit(V a) { float r = 1.0f / std::sqrt(dot(a, a)); return mul(a, r); }
static void acc(V& a, V b) { a.x += b.x; a.y += b.y; a.z += b.z; }

// offsetRayOrigin (include/core/ray.cuh:10-21): push the point off the
// surface by 32 float epsilons of its magnitude, then one more ulp.
static V nudge(V p, V n, V d, float t) {
    float m = std::fmax(std::fmax(1.0f, std::fabs(t)), std::fmax(std::fabs(p.x), std::fmax(std::fabs(p.y), std::fabs(p.z))));
    float s = dot(d, n) >= 0.0f ? 1.0f : -1.0f;
    V o = mul(n, s * 32.0f * 1.1920928955078125e-7f * m);
    V r = add(p, o);
    if (o.x != 0) r.x = std::nextafter(r.x, o.x > 0 ? INFINITY : -INFINITY);
    if (o.y != 0) r.y = std::nextafter(r.y, o.y > 0 ? INFINITY : -INFINITY);
    if (o.z != 0) r.z = std::nextafter(r.z, o.z > 0 ? INFINITY : -INFINITY);
    return r;
}

// ------------------------------------------------------------------- RNG
struct Rng {
    uint64_t s = 0;
    uint32_t kind = 0;
    float next() {
        uint32_t v;
        if (kind == 0) {
            uint32_t x = uint32_t(s);
            x ^= x << 13;
            x ^= x >> 17;
            x ^= x << 5;
            s = x;
            v = x;
        } else {
            uint64_t o = s;
            s = o * 6364136223846793005ull + 1442695040888963407ull;
            uint32_t xs = uint32_t(((o >> 18u) ^ o) >> 27u);
            uint32_t rot = uint32_t(o >> 59u);
            v = (xs >> rot) | (xs << ((32u - rot) & 31u));
        }
        return float(v >> 8) * 0x1.0p-24f;
    }
};
static Rng seed_rng(uint64_t key, uint32_t kind) {
    Rng r;
    r.kind = kind;
    if (kind == 0) {
        uint32_t z = uint32_t(key) * 747796405u + 2891336453u;
        r.s = z == 0 ? 1u : z;
    } else {
        uint64_t z = key + 0x9e3779b97f4a7c15ull;
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        r.s = z ^ (z >> 31);
    }
    return r;
}
static uint64_t pixel_key(uint32_t pixel, uint32_t sample, uint32_t kind) {
    return kind == 0 ? uint64_t(pixel ^ (sample * 0x9e3779b9u)) : ((uint64_t(sample) << 32) | pixel);
}
static uint64_t photon_key(uint32_t photon, uint32_t seed, uint32_t kind) {
    return kind == 0 ? uint64_t(seed ^ (photon * 0x9e3779b9u)) : ((uint64_t(seed) << 32) | photon);
}

// ----------------------------------------------------------------- scene
struct Tri {
    V a, b, c, na, nb, nc;
    uint32_t mat = 0, light = NONE;
    bool normals = false;
};
struct Node {
    float lo[3], hi[3];
    uint32_t left, right;
};
struct Tree {
    std::vector<Node> nodes;  // root last; leaf: left == NONE, right = primitive
};
struct Mat {
    uint32_t type = 0;
    V albedo, emission;
    float roughness = 0, ior = 1, metallic = 0, dispersion = 0;
    V att_color;
    float att_distance = 0, density = 1, opacity = 1, cutoff = 0.5f;
    bool masked = false;
};
struct Inst {
    V l2w[3], w2l[3], t;
    uint32_t mesh, override_mat, light_offset;
};
struct Light {
    V a, b, c, n;
    float area, pdf, alias_p;
    uint32_t mat, alias;
};
struct Punct {
    uint32_t type;
    V pos, dir, intensity;
    float range, inner, outer;
};
struct Env {
    uint32_t w = 0, h = 0;
    std::vector<float> px;  // rgba
    std::vector<float> prob, alias_p;
    std::vector<uint32_t> alias;
    float intensity = 1, rotation = 0;
    bool on = false;
};
struct Scene {
    std::vector<V> sp_c;
    std::vector<float> sp_r;
    std::vector<uint32_t> sp_m, direct_spheres, direct_insts;
    std::vector<std::pair<bool, uint32_t>> leaves;  // (is sphere, index)
    Tree tlas;
    std::vector<std::vector<Tri>> meshes;
    std::vector<Tree> blas;
    std::vector<Inst> insts;
    std::vector<Tri> statics, directs;
    Tree direct_tree;
    bool direct_tree_on = false;
    std::vector<Mat> mats;
    std::vector<Light> lights;
    std::vector<Punct> punct;
    uint32_t directional = 0;
    Env env;
    bool black = false, ignore_occ = false;
};

static Tree make_tree(std::vector<wf::BvhBox>& boxes) {
    std::vector<wf::BvhBinaryNode> bin;
    wf::build_binary_bvh(boxes.data(), uint32_t(boxes.size()), bin, 0);
    Tree t;
    t.nodes.resize(bin.size());
    for (size_t i = 0; i < bin.size(); ++i) {
        for (int k = 0; k < 3; ++k) { t.nodes[i].lo[k] = bin[i].box.lo[k]; t.nodes[i].hi[k] = bin[i].box.hi[k]; }
        t.nodes[i].left = bin[i].left;
        t.nodes[i].right = bin[i].right;
    }
    return t;
}
static wf::BvhBox tri_box(const Tri& t) {
    wf::BvhBox b;
    const V* v[3] = {&t.a, &t.b, &t.c};
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (auto* p : v) {
        float c[3] = {p->x, p->y, p->z};
        for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], c[k]); hi[k] = std::max(hi[k], c[k]); }
    }
    for (int k = 0; k < 3; ++k) { b.lo[k] = lo[k]; b.hi[k] = hi[k]; }
    return b;
}
static Tri to_tri(const wf_triangle& t) {
    Tri r;
    r.a = mk3(t.v0); r.b = mk3(t.v1); r.c = mk3(t.v2);
    r.na = mk3(t.n0); r.nb = mk3(t.n1); r.nc = mk3(t.n2);
    r.mat = t.material;
    r.normals = t.has_vertex_normals != 0;
    return r;
}
static V l2w(const Inst& in, V v) { return add(add(mul(in.l2w[0], v.x), mul(in.l2w[1], v.y)), mul(in.l2w[2], v.z)); }
static V w2l(const Inst& in, V v) { return add(add(mul(in.w2l[0], v.x), mul(in.w2l[1], v.y)), mul(in.w2l[2], v.z)); }

// environmentSolidAngle (environment.cuh:35-39).
static float solid_angle(uint32_t row, uint32_t w, uint32_t h) {
    const double pi = 3.14159265358979323846;
    return float((4.0 * pi / w) * m_sin(pi * (row + 0.5) / h) * m_sin(pi / (2.0 * h)));
}

// Light alias table (scene.cu:82-121): float Vose method.
static void alias_lights(std::vector<Light>& lights, const std::vector<float>& weight) {
    if (lights.empty()) return;
    float total = 0.0f;
    for (float w : weight) total += w;
    size_t n = lights.size();
    std::vector<float> sc(n);
    std::vector<uint32_t> lo, hi;
    for (uint32_t i = 0; i < n; ++i) {
        lights[i].pdf = weight[i] / total;
        sc[i] = lights[i].pdf * n;
        if (sc[i] < 1.0f) lo.push_back(i); else hi.push_back(i);
        lights[i].alias_p = 1.0f;
        lights[i].alias = i;
    }
    while (!lo.empty() && !hi.empty()) {
        uint32_t l = lo.back(), g = hi.back();
        lo.pop_back();
        hi.pop_back();
        lights[l].alias_p = sc[l];
        lights[l].alias = g;
        sc[g] = sc[g] + sc[l] - 1.0f;
        if (sc[g] < 1.0f) lo.push_back(g); else hi.push_back(g);
    }
    for (uint32_t i : lo) { lights[i].alias_p = 1.0f; lights[i].alias = i; }
    for (uint32_t i : hi) { lights[i].alias_p = 1.0f; lights[i].alias = i; }
}

static void push_light(Scene& s, std::vector<float>& weights, V a, V b, V c, uint32_t mat, const Mat& m) {
    Light l;
    l.a = a; l.b = b; l.c = c;
    l.n = unit(cross(sub(b, a), sub(c, a)));
    l.area = 0.5f * len(cross(sub(b, a), sub(c, a)));
    l.mat = mat;
    l.pdf = 0; l.alias_p = 1; l.alias = 0;
    s.lights.push_back(l);
    weights.push_back(l.area * (0.2126f * m.emission.x + 0.7152f * m.emission.y + 0.0722f * m.emission.z));
}

// buildEnvironmentDistribution (environment.cpp:10-64).
static bool build_env(Env& e, const wf_environment* in) {
    uint64_t n = uint64_t(in->width) * in->height;
    if (n == 0) return false;
    e.w = in->width;
    e.h = in->height;
    e.px.assign(in->rgba, in->rgba + 4 * n);
    for (uint64_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k)
            if (!std::isfinite(e.px[4 * i + k]) || e.px[4 * i + k] < 0) return false;
    std::vector<double> w(n);
    double total = 0;
    const double f[3] = {0.125, 0.75, 0.125};
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t x = i % e.w, y = i / e.w;
        uint32_t cx[3] = {x ? x - 1 : e.w - 1, x, x + 1 < e.w ? x + 1 : 0};
        uint32_t cy[3] = {y ? y - 1 : 0, y, y + 1 < e.h ? y + 1 : e.h - 1};
        double a = 0;
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
                const float* p = &e.px[4 * (uint64_t(cy[r]) * e.w + cx[c])];
                a += f[r] * f[c] * (0.2126 * double(p[0]) + 0.7152 * double(p[1]) + 0.0722 * double(p[2]));
            }
        w[i] = a * solid_angle(y, e.w, e.h);
        total += w[i];
    }
    const double four_pi = 12.5663706143591729538;
    e.prob.resize(n);
    e.alias_p.assign(n, 1.0f);
    e.alias.resize(n);
    double sum = 0;
    for (uint32_t i = 0; i < n; ++i) {
        double u = solid_angle(i / e.w, e.w, e.h) / four_pi;
        e.prob[i] = float(total > 0 ? .99 * w[i] / total + .01 * u : u);
        sum += e.prob[i];
    }
    std::vector<uint32_t> lo, hi;
    for (uint32_t i = 0; i < n; ++i) {
        e.prob[i] /= sum;
        w[i] = double(e.prob[i]) * n;
        e.alias[i] = i;
        if (w[i] < 1.0) lo.push_back(i); else hi.push_back(i);
    }
    while (!lo.empty() && !hi.empty()) {
        uint32_t l = lo.back(), g = hi.back();
        lo.pop_back();
        hi.pop_back();
        e.alias_p[l] = float(w[l]);
        e.alias[l] = g;
        w[g] += w[l] - 1;
        if (w[g] < 1.0) lo.push_back(g); else hi.push_back(g);
    }
    for (uint32_t i : lo) { e.alias_p[i] = 1; e.alias[i] = i; }
    for (uint32_t i : hi) { e.alias_p[i] = 1; e.alias[i] = i; }
    e.intensity = in->intensity;
    e.rotation = std::fmod(in->rotation_degrees, 360.0f) * (3.14159265359f / 180.0f);
    e.on = true;
    return true;
}

static Scene* build_scene(const wf_scene_desc* d, const wf_environment* env) {
    auto s = std::make_unique<Scene>();
    for (uint32_t i = 0; i < d->material_count; ++i) {
        const wf_material& m = d->materials[i];
        Mat r;
        r.type = m.type;
        r.albedo = mk3(m.albedo);
        r.emission = mk3(m.emission);
        r.roughness = m.roughness;
        r.ior = m.ior;
        r.metallic = m.metallic;
        r.dispersion = m.dispersion;
        r.att_color = mk3(m.attenuation_color);
        r.att_distance = m.attenuation_distance;
        r.density = m.volume_density;
        r.opacity = m.opacity;
        r.cutoff = m.alpha_cutoff;
        r.masked = m.alpha_masked != 0;
        s->mats.push_back(r);
    }
    auto emissive = [&](uint32_t m) { return s->mats[m].type == WF_MAT_EMISSIVE; };
    bool reg = d->register_triangle_lights != 0;
    // meshes with per-mesh light numbering (scene_host.cpp:77-86)
    std::vector<uint32_t> mesh_lights(d->mesh_count, 0);
    for (uint32_t m = 0; m < d->mesh_count; ++m) {
        std::vector<Tri> tris;
        uint32_t local = 0;
        for (uint32_t i = 0; i < d->meshes[m].triangle_count; ++i) {
            Tri t = to_tri(d->meshes[m].triangles[i]);
            t.light = reg && emissive(t.mat) ? local++ : NONE;
            tris.push_back(t);
        }
        mesh_lights[m] = local;
        s->meshes.push_back(std::move(tris));
    }
    std::vector<float> weights;
    for (uint32_t i = 0; i < d->instance_count; ++i) {
        const wf_instance& w = d->instances[i];
        Inst in;
        for (int k = 0; k < 3; ++k) { in.l2w[k] = mk3(w.local_to_world[k]); in.w2l[k] = mk3(w.world_to_local[k]); }
        in.t = mk3(w.translation);
        in.mesh = w.mesh;
        in.override_mat = w.material_override;
        in.light_offset = 0;
        s->insts.push_back(in);
    }
    if (reg) {  // mesh lights per instance (scene_host.cpp:88-105)
        for (const Inst& in : s->insts)
            for (const Tri& t : s->meshes[in.mesh])
                if (t.light != NONE)
                    push_light(*s, weights, add(l2w(in, t.a), in.t), add(l2w(in, t.b), in.t), add(l2w(in, t.c), in.t),
                               t.mat, s->mats[t.mat]);
    }
    for (uint32_t i = 0; i < d->static_triangle_count; ++i) {
        Tri t = to_tri(d->static_triangles[i]);
        if (reg && emissive(t.mat)) {  // scene_host.cpp:60-75
            t.light = uint32_t(s->lights.size());
            push_light(*s, weights, t.a, t.b, t.c, t.mat, s->mats[t.mat]);
        }
        s->statics.push_back(t);
    }
    alias_lights(s->lights, weights);
    uint32_t offset = 0;
    for (Inst& in : s->insts) {
        in.light_offset = offset;
        offset += mesh_lights[in.mesh];
    }
    // BLAS only for meshes referenced by an accelerated instance (scene.cu:124-150).
    s->blas.resize(d->mesh_count);
    for (uint32_t m = 0; m < d->mesh_count; ++m) {
        bool need = false;
        for (uint32_t i = 0; i < d->instance_count; ++i)
            need |= d->instances[i].mesh == m && d->instances[i].accel == WF_ACCEL_BVH;
        if (!need || s->meshes[m].empty()) continue;
        std::vector<wf::BvhBox> boxes;
        for (const Tri& t : s->meshes[m]) boxes.push_back(tri_box(t));
        s->blas[m] = make_tree(boxes);
    }
    // TLAS over accelerated spheres, then accelerated instances (scene.cu:175-239).
    std::vector<wf::BvhBox> boxes;
    for (uint32_t i = 0; i < d->sphere_count; ++i) {
        const wf_sphere& sp = d->spheres[i];
        s->sp_c.push_back(mk3(sp.center));
        s->sp_r.push_back(sp.radius);
        s->sp_m.push_back(sp.material);
        if (sp.accel == WF_ACCEL_DIRECT) {
            s->direct_spheres.push_back(i);
            continue;
        }
        float r = std::fabs(sp.radius);
        wf::BvhBox b;
        for (int k = 0; k < 3; ++k) {
            b.lo[k] = std::nextafter(sp.center[k] - r, -INFINITY);
            b.hi[k] = std::nextafter(sp.center[k] + r, INFINITY);
        }
        boxes.push_back(b);
        s->leaves.push_back({true, i});
    }
    for (uint32_t i = 0; i < d->instance_count; ++i) {
        const Inst& in = s->insts[i];
        if (d->instances[i].accel == WF_ACCEL_DIRECT) {
            s->direct_insts.push_back(i);
            continue;
        }
        if (s->meshes[in.mesh].empty()) continue;
        const Node& root = s->blas[in.mesh].nodes.back();
        wf::BvhBox w;
        for (int k = 0; k < 3; ++k) { w.lo[k] = INFINITY; w.hi[k] = -INFINITY; }
        for (uint32_t c = 0; c < 8; ++c) {
            V p = mk((c & 1) ? root.hi[0] : root.lo[0], (c & 2) ? root.hi[1] : root.lo[1], (c & 4) ? root.hi[2] : root.lo[2]);
            V q = add(l2w(in, p), in.t);
            w.lo[0] = std::fmin(w.lo[0], q.x); w.lo[1] = std::fmin(w.lo[1], q.y); w.lo[2] = std::fmin(w.lo[2], q.z);
            w.hi[0] = std::fmax(w.hi[0], q.x); w.hi[1] = std::fmax(w.hi[1], q.y); w.hi[2] = std::fmax(w.hi[2], q.z);
        }
        boxes.push_back(w);
        s->leaves.push_back({false, i});
    }
    if (!boxes.empty()) s->tlas = make_tree(boxes);
    for (uint32_t i = 0; i < d->triangle_count; ++i) s->directs.push_back(to_tri(d->triangles[i]));
    if (!s->directs.empty() && d->mesh_count == 0) {  // scene.cu:361-375
        std::vector<wf::BvhBox> b;
        for (const Tri& t : s->directs) b.push_back(tri_box(t));
        s->direct_tree = make_tree(b);
        s->direct_tree_on = true;
    }
    for (int pass = 0; pass < 2; ++pass)  // directional prefix (scene.cu:346-351)
        for (uint32_t i = 0; i < d->punctual_light_count; ++i) {
            const wf_punctual_light& l = d->punctual_lights[i];
            if ((l.type == WF_LIGHT_DIRECTIONAL) != (pass == 0)) continue;
            s->punct.push_back(Punct{l.type, mk3(l.position), mk3(l.direction), mk3(l.intensity), l.range,
                                     l.inner_cone_cos, l.outer_cone_cos});
            if (pass == 0) ++s->directional;
        }
    s->black = d->black_background != 0;
    s->ignore_occ = d->ignore_direct_light_occlusion != 0;
    if (env && env->width && !build_env(s->env, env)) return nullptr;
    return s.release();
}

// ------------------------------------------------------------- traversal
struct Ray {
    V o, d;
};
struct Best {
    float t = 1e30f;
    int mat = -1;
    uint32_t kind = 0, prim = NONE, inst = NONE, sphere = NONE;
    float u = 0, v = 0;
};

static bool hit_sphere(const Ray& r, V c, float rad, float& t) {  // device_traversal.cuh:24-53
    V oc = sub(r.o, c);
    float a = dot(r.d, r.d);
    float b = 2.0f * dot(oc, r.d);
    float cc = dot(oc, oc) - rad * rad;
    float disc = b * b - 4.0f * a * cc;
    if (disc < 0.0f) return false;
    float q = std::sqrt(disc);
    float t0 = (-b - q) / (2.0f * a), t1 = (-b + q) / (2.0f * a);
    if (t0 > T_MIN) { t = t0; return true; }
    if (t1 > T_MIN) { t = t1; return true; }
    return false;
}

static bool hit_tri(const Ray& r, const Tri& tr, float& t, float& u, float& v) {  // :55-91
    V e1 = sub(tr.b, tr.a), e2 = sub(tr.c, tr.a);
    V p = cross(r.d, e2);
    float det = dot(e1, p);
    float scale = std::fabs(e1.x) * (std::fabs(r.d.y * e2.z) + std::fabs(r.d.z * e2.y)) +
                  std::fabs(e1.y) * (std::fabs(r.d.z * e2.x) + std::fabs(r.d.x * e2.z)) +
                  std::fabs(e1.z) * (std::fabs(r.d.x * e2.y) + std::fabs(r.d.y * e2.x));
    if (!std::isfinite(det) || std::fabs(det) <= 8.0f * FLT_EPSILON * scale) return false;
    float inv = 1.0f / det;
    V s = sub(r.o, tr.a);
    u = dot(s, p) * inv;
    if (u < 0.0f || u > 1.0f) return false;
    V q = cross(s, e1);
    v = dot(r.d, q) * inv;
    if (v < 0.0f || u + v > 1.0f) return false;
    t = dot(e2, q) * inv;
    return t > T_MIN;
}

static bool box(const Ray& r, V inv, const Node& n, float limit, float& near_t) {  // :182-197
    float tx0 = (n.lo[0] - r.o.x) * inv.x, tx1 = (n.hi[0] - r.o.x) * inv.x;
    float ty0 = (n.lo[1] - r.o.y) * inv.y, ty1 = (n.hi[1] - r.o.y) * inv.y;
    float tz0 = (n.lo[2] - r.o.z) * inv.z, tz1 = (n.hi[2] - r.o.z) * inv.z;
    float lo = std::fmax(std::fmin(tx0, tx1), std::fmax(std::fmin(ty0, ty1), std::fmin(tz0, tz1)));
    float hi = std::fmin(std::fmax(tx0, tx1), std::fmin(std::fmax(ty0, ty1), std::fmax(tz0, tz1)));
    near_t = lo;
    return hi >= std::fmax(lo, T_MIN) && lo < limit;
}

static bool rejected(const Scene& s, uint32_t m) { return s.mats[m].masked && s.mats[m].opacity < s.mats[m].cutoff; }

// Stack traversal of a binary tree: the popped node's box is tested against
// the current limit, children are pushed far then near (near = strictly
// smaller entry distance, ties to the right child).  `leaf` returns true to
// stop the traversal (any-hit).
template <typename Leaf>
static bool walk(const Tree& tree, const Ray& r, const float& limit, Leaf&& leaf) {
    if (tree.nodes.empty()) return false;
    V inv = mk(1.0f / r.d.x, 1.0f / r.d.y, 1.0f / r.d.z);
    uint32_t stack[64];
    int n = 1;
    stack[0] = uint32_t(tree.nodes.size() - 1);
    while (n > 0) {
        const Node& node = tree.nodes[stack[--n]];
        float nt;
        if (!box(r, inv, node, limit, nt)) continue;
        if (node.left == NONE) {
            if (leaf(node.right)) return true;
            continue;
        }
        float tl, trr;
        bool hl = box(r, inv, tree.nodes[node.left], limit, tl);
        bool hr = box(r, inv, tree.nodes[node.right], limit, trr);
        if (hl && hr) {
            bool left_near = tl < trr;
            stack[n++] = left_near ? node.right : node.left;
            stack[n++] = left_near ? node.left : node.right;
        } else if (hl) {
            stack[n++] = node.left;
        } else if (hr) {
            stack[n++] = node.right;
        }
    }
    return false;
}

static void take_tri(Best& b, float t, float u, float v, uint32_t mat, uint32_t kind, uint32_t prim, uint32_t inst) {
    b.t = t; b.u = u; b.v = v;
    b.mat = int(mat);
    b.kind = kind; b.prim = prim; b.inst = inst;
}

static void visit_instance(const Scene& s, const Ray& wr, uint32_t i, Best& b, bool use_tree) {  // :802-834
    const Inst& in = s.insts[i];
    Ray r{w2l(in, sub(wr.o, in.t)), w2l(in, wr.d)};
    float before = b.t;
    const std::vector<Tri>& tris = s.meshes[in.mesh];
    auto test = [&](uint32_t k) {
        float t, u, v;
        if (!hit_tri(r, tris[k], t, u, v) || !(t < b.t)) return false;
        uint32_t m = in.override_mat == NONE ? tris[k].mat : in.override_mat;
        if (rejected(s, m)) return false;
        take_tri(b, t, u, v, m, WF_HIT_MESH, k, i);
        return false;
    };
    if (use_tree && !s.blas[in.mesh].nodes.empty())
        walk(s.blas[in.mesh], r, b.t, test);
    else
        for (uint32_t k = 0; k < tris.size(); ++k) test(k);
    if (b.t < before) b.sphere = NONE;
}

static void visit_sphere(const Scene& s, const Ray& r, uint32_t i, Best& b) {  // :789-800
    float t;
    if (!hit_sphere(r, s.sp_c[i], s.sp_r[i], t) || t > b.t) return;
    if (t == b.t && i >= b.sphere) return;
    b.t = t;
    b.mat = int(s.sp_m[i]);
    b.kind = WF_HIT_SPHERE;
    b.prim = i;
    b.inst = NONE;
    b.sphere = i;
}

static Best closest(const Scene& s, const Ray& r) {  // traceRay, :1115-1150
    Best b;
    for (uint32_t i : s.direct_spheres) visit_sphere(s, r, i, b);
    for (uint32_t i : s.direct_insts) visit_instance(s, r, i, b, false);
    for (uint32_t k = 0; k < s.statics.size(); ++k) {
        float t, u, v;
        if (!hit_tri(r, s.statics[k], t, u, v) || !(t < b.t) || rejected(s, s.statics[k].mat)) continue;
        take_tri(b, t, u, v, s.statics[k].mat, WF_HIT_STATIC_TRIANGLE, k, NONE);
        b.sphere = NONE;
    }
    walk(s.tlas, r, b.t, [&](uint32_t leaf) {
        if (s.leaves[leaf].first) visit_sphere(s, r, s.leaves[leaf].second, b);
        else visit_instance(s, r, s.leaves[leaf].second, b, true);
        return false;
    });
    if (!s.directs.empty()) {
        float before = b.t;
        auto test = [&](uint32_t k) {
            float t, u, v;
            if (!hit_tri(r, s.directs[k], t, u, v) || !(t < b.t) || rejected(s, s.directs[k].mat)) return false;
            take_tri(b, t, u, v, s.directs[k].mat, WF_HIT_TRIANGLE, k, NONE);
            return false;
        };
        if (s.direct_tree_on) walk(s.direct_tree, r, b.t, test);
        else for (uint32_t k = 0; k < s.directs.size(); ++k) test(k);
        if (b.t < before) b.sphere = NONE;
    }
    return b;
}

static bool blocked(const Scene& s, const Ray& r, float limit) {  // isOccluded, :1035-1113
    float t;
    for (uint32_t i : s.direct_spheres)
        if (hit_sphere(r, s.sp_c[i], s.sp_r[i], t) && t < limit) return true;
    auto inst_any = [&](uint32_t i, bool tree) {
        const Inst& in = s.insts[i];
        Ray lr{w2l(in, sub(r.o, in.t)), w2l(in, r.d)};
        const std::vector<Tri>& tris = s.meshes[in.mesh];
        auto test = [&](uint32_t k) {
            float tt, u, v;
            if (!hit_tri(lr, tris[k], tt, u, v) || !(tt < limit)) return false;
            return !rejected(s, in.override_mat == NONE ? tris[k].mat : in.override_mat);
        };
        if (tree && !s.blas[in.mesh].nodes.empty()) return walk(s.blas[in.mesh], lr, limit, test);
        for (uint32_t k = 0; k < tris.size(); ++k)
            if (test(k)) return true;
        return false;
    };
    for (uint32_t i : s.direct_insts)
        if (inst_any(i, false)) return true;
    for (const Tri& tr : s.statics) {
        float u, v;
        if (hit_tri(r, tr, t, u, v) && t < limit && !rejected(s, tr.mat)) return true;
    }
    if (walk(s.tlas, r, limit, [&](uint32_t leaf) {
            float tt;
            if (s.leaves[leaf].first) {
                uint32_t i = s.leaves[leaf].second;
                return hit_sphere(r, s.sp_c[i], s.sp_r[i], tt) && tt < limit;
            }
            return inst_any(s.leaves[leaf].second, true);
        }))
        return true;
    if (!s.directs.empty()) {
        auto test = [&](uint32_t k) {
            float tt, u, v;
            return hit_tri(r, s.directs[k], tt, u, v) && tt < limit && !rejected(s, s.directs[k].mat);
        };
        if (s.direct_tree_on) return walk(s.direct_tree, r, limit, test);
        for (uint32_t k = 0; k < s.directs.size(); ++k)
            if (test(k)) return true;
    }
    return false;
}

struct Hit {
    float t;
    V p, gn, n;
    uint32_t mat, light;
};

static V face(V n, V d, bool ff) { return ff && dot(n, d) > 0.0f ? neg(n) : n; }
static V tri_gn(const Tri& t) { return unit(cross(sub(t.b, t.a), sub(t.c, t.a))); }
static V tri_sn(const Tri& t, float u, float v) {
    if (!t.normals) return tri_gn(t);
    float w = 1.0f - u - v;
    return unit(add(add(mul(t.na, w), mul(t.nb, u)), mul(t.nc, v)));
}

static bool finish(const Scene& s, const Ray& r, const Best& b, Hit& h) {  // attributes, :104-180,824-832,1152-1184
    if (b.mat < 0) return false;
    h.t = b.t;
    h.mat = uint32_t(b.mat);
    if (b.kind == WF_HIT_SPHERE) {
        V at = add(r.o, mul(r.d, b.t));
        h.n = unit(sub(at, s.sp_c[b.prim]));
        h.gn = h.n;
        h.light = NONE;
    } else if (b.kind == WF_HIT_MESH) {
        const Inst& in = s.insts[b.inst];
        const Tri& t = s.meshes[in.mesh][b.prim];
        V ld = w2l(in, r.d);
        bool ff = s.mats[h.mat].type != WF_MAT_DIELECTRIC;
        V gn = face(tri_gn(t), ld, ff), n = face(tri_sn(t, b.u, b.v), ld, ff);
        auto xform = [&](V v) { return unit(mk(dot(in.w2l[0], v), dot(in.w2l[1], v), dot(in.w2l[2], v))); };
        h.gn = xform(gn);
        h.n = xform(n);
        h.light = in.override_mat == NONE ? t.light : NONE;
        if (h.light != NONE) h.light += in.light_offset;
    } else {
        const Tri& t = b.kind == WF_HIT_STATIC_TRIANGLE ? s.statics[b.prim] : s.directs[b.prim];
        bool ff = s.mats[h.mat].type != WF_MAT_DIELECTRIC;
        h.gn = face(tri_gn(t), r.d, ff);
        h.n = face(tri_sn(t, b.u, b.v), r.d, ff);
        h.light = b.kind == WF_HIT_STATIC_TRIANGLE ? t.light : NONE;
    }
    h.p = add(r.o, mul(r.d, b.t));
    return true;
}

// ------------------------------------------------------------ environment
static V rot_env(V d, float a) {  // environment.cuh:19-22
    float c = m_cosf(a), s = m_sinf(a);
    return mk(c * d.x + s * d.z, d.y, -s * d.x + c * d.z);
}
static void env_uv(const Env& e, V w, float& u, float& v) {  // :26-33
    V d = rot_env(w, -e.rotation);
    const float pi = 3.14159265359f;
    u = m_atan2f(d.z, d.x) / (2.0f * pi) + 0.5f;
    u -= std::floor(u);
    float vv = m_atan2f(std::sqrt(d.x * d.x + d.z * d.z), d.y) / pi;
    v = std::fmin(1.0f, std::fmax(0.0f, vv));
}
static float env_pdf(const Env& e, V d) {  // :46-50
    if (!e.w || !e.h || e.prob.empty()) return 0.0f;
    float u, v;
    env_uv(e, d, u, v);
    uint32_t x = uint32_t(u * e.w), y = uint32_t(v * e.h);
    uint32_t i = (y < e.h ? y : e.h - 1) * e.w + (x < e.w ? x : e.w - 1);
    return e.prob[i] / solid_angle(i / e.w, e.w, e.h);
}
static V env_lookup(const Env& e, V d) {  // environmentRadiance + bilinear wrap/clamp filter
    float u, v;
    env_uv(e, d, u, v);
    float tx = u * e.w - .5f, ty = v * e.h - .5f;
    int x = int(std::floor(tx)), y = int(std::floor(ty));
    float fx = tx - x, fy = ty - y;
    V out;
    for (int j = 0; j < 2; ++j)
        for (int i = 0; i < 2; ++i) {
            int xx = ((x + i) % int(e.w) + int(e.w)) % int(e.w);
            int yy = std::min(std::max(y + j, 0), int(e.h) - 1);
            const float* p = &e.px[4 * (size_t(yy) * e.w + xx)];
            float w = (i ? fx : 1 - fx) * (j ? fy : 1 - fy);
            out.x += w * p[0];
            out.y += w * p[1];
            out.z += w * p[2];
        }
    return mul(out, e.intensity);
}
struct EnvPick {
    V d;
    float pdf;
};
static EnvPick env_sample(const Env& e, Rng& rng) {  // samplePathEnvironment + sampleEnvironment
    float coarse = rng.next(), fine = rng.next();
    double cand = double(coarse) + double(fine) * (1.0 / 16777216.0);
    float coin = rng.next(), lon = rng.next(), lat = rng.next();
    uint32_t n = e.w * e.h;
    uint32_t i = uint32_t(cand * n);
    if (i >= n) i = n - 1;
    if (coin >= e.alias_p[i]) i = e.alias[i];
    uint32_t x = i % e.w, y = i / e.w;
    const double pi = 3.14159265358979323846;
    double u = (x + std::fmin(1.0f - 1.0e-7f, std::fmax(1.0e-7f, lon))) / e.w;
    double jit = std::fmin(1.0f - 1.0e-7f, std::fmax(1.0e-7f, lat));
    double c = (1.0 - jit) * m_cos(pi * y / e.h) + jit * m_cos(pi * (y + 1.0) / e.h);
    double sn = std::sqrt(std::fmax(0.0, 1.0 - c * c));
    double phi = (u - 0.5) * 2 * pi;
    V local = mk(float(sn * m_cos(phi)), float(c), float(sn * m_sin(phi)));
    return EnvPick{rot_env(local, e.rotation), e.prob[i] / solid_angle(y, e.w, e.h)};
}

// ------------------------------------------------------------------ BSDFs
static float mis(float a, float b) { float a2 = a * a, b2 = b * b; return a2 / (a2 + b2); }
static V cos_hemi(V n, Rng& rng) {  // device_sampling.cuh:6-25
    float u1 = rng.next(), u2 = rng.next();
    float rad = std::sqrt(u1), phi = 6.28318530718f * u2;
    float x = rad * m_cosf(phi), y = rad * m_sinf(phi), z = std::sqrt(1.0f - u1);
    V helper = std::fabs(n.x) > 0.1f ? mk(0, 1, 0) : mk(1, 0, 0);
    V t = unit(cross(helper, n));
    V b = cross(n, t);
    return unit(add(add(mul(t, x), mul(b, y)), mul(n, z)));
}
static V reflect(V i, V n) { return sub(i, mul(n, 2.0f * dot(i, n))); }
static V refract(V i, V n, float eta) {
    float c = std::fmin(dot(neg(i), n), 1.0f);
    V perp = mul(add(i, mul(n, c)), eta);
    V par = mul(n, -std::sqrt(std::fmax(0.0f, 1.0f - len2(perp))));
    return add(perp, par);
}
static float fresnel(float c, float eta) {  // dielectricReflectance
    if (eta == 1.0f) return 0.0f;
    c = std::fmin(1.0f, std::fmax(0.0f, c));
    float s2 = eta * eta * std::fmax(0.0f, 1.0f - c * c);
    if (s2 >= 1.0f) return 1.0f;
    float ct = std::sqrt(1.0f - s2);
    float rs = (eta * c - ct) / (eta * c + ct), rp = (c - eta * ct) / (c + eta * ct);
    return 0.5f * (rs * rs + rp * rp);
}
struct Boundary {
    V refl, trans;
    float eta, R;
    bool front;
};
static Boundary interface(V i, V gn, V sn, float ior) {  // dielectricInterface
    Boundary b;
    b.front = dot(i, gn) < 0.0f;
    V facing = b.front ? gn : neg(gn);
    if (dot(sn, gn) < 0.0f) sn = neg(sn);
    V n = b.front ? sn : neg(sn);
    b.eta = b.front ? 1.0f / ior : ior;
    if (dot(i, n) >= 0.0f) n = facing;
    b.R = fresnel(dot(neg(i), n), b.eta);
    b.refl = reflect(i, n);
    b.trans = refract(i, n, b.eta);
    if (dot(b.refl, facing) <= 0.0f || (b.R < 1.0f && dot(b.trans, facing) >= 0.0f)) {
        n = facing;
        b.R = fresnel(dot(neg(i), n), b.eta);
        b.refl = reflect(i, n);
        b.trans = refract(i, n, b.eta);
    }
    return b;
}
// GGX metal lobe of the specular-glossiness model with diffuse = 0
// (specular_glossiness.cuh:13-80).
static float vmax(V v) { return std::fmax(v.x, std::fmax(v.y, v.z)); }
static float ggx_prob(V f0, V dif) {
    float sp = vmax(f0), df = vmax(dif) * (1.0f - sp);
    return std::fmin(0.95f, std::fmax(0.05f, sp / std::fmax(1.0e-6f, sp + df)));
}
static float ggx_alpha(float r) { float a = std::fmax(0.02f, r); return a * a; }
static float ggx_d(float nh, float a) {
    float a2 = a * a, den = (1.0f - nh * nh) + a2 * nh * nh;
    return a2 / (3.14159265359f * den * den);
}
static float ggx_g1(float c, float a) { return 2.0f * c / (c + std::sqrt(a * a + (1.0f - a * a) * c * c)); }
static V ggx_eval(V dif, V f0, float rough, V n, V o, V i, float& pdf) {
    pdf = 0.0f;
    float nv = dot(n, o), nl = dot(n, i);
    V sum = add(o, i);
    if (nv <= 0.0f || nl <= 0.0f || len2(sum) < 1.0e-12f) return V();
    V h = unit(sum);
    float nh = std::fmin(1.0f, std::fmax(0.0f, dot(n, h)));
    float vh = std::fmin(1.0f, std::fmax(1.0e-8f, dot(o, h)));
    float a = ggx_alpha(rough), d = ggx_d(nh, a), p = ggx_prob(f0, dif);
    pdf = (1.0f - p) * nl * 0.31830988618f + p * d * nh / (4.0f * vh);
    float sch = m_powf(1.0f - vh, 5.0f);
    V fr = add(f0, mul(sub(mk(1, 1, 1), f0), sch));
    V diff = mul(dif, (1.0f - vmax(f0)) * 0.31830988618f);
    float g = ggx_g1(nv, a) * ggx_g1(nl, a);
    return add(diff, mul(fr, d * g / (4.0f * nv * nl)));
}
static V basis(V n, float x, float y, float z) {
    V helper = std::fabs(n.x) > 0.1f ? mk(0, 1, 0) : mk(1, 0, 0);
    V t = unit(cross(helper, n));
    return unit(add(add(mul(t, x), mul(cross(n, t), y)), mul(n, z)));
}
static V ggx_sample(V dif, V f0, float rough, V n, V o, float choice, float u, float v) {
    float phi = 6.28318530718f * v;
    if (choice < ggx_prob(f0, dif)) {
        float a = ggx_alpha(rough);
        float c = std::sqrt((1.0f - u) / (1.0f + (a * a - 1.0f) * u));
        float sn = std::sqrt(std::fmax(0.0f, 1.0f - c * c));
        V h = basis(n, sn * m_cosf(phi), sn * m_sinf(phi), c);
        return sub(mul(h, 2.0f * dot(o, h)), o);
    }
    float rad = std::sqrt(u);
    return basis(n, rad * m_cosf(phi), rad * m_sinf(phi), std::sqrt(1.0f - u));
}

// ------------------------------------------------------------------ paths
struct Cfg {
    uint32_t width, height, depth, rr, rng, debug;
    float clamp, gather;
    V cam_p, cam_f, cam_r, cam_u;
    float aspect, tan_half;
};
struct PhotonMap;
struct PathCtx {
    const Scene& s;
    const Cfg& c;
    const PhotonMap* pm;
};
struct Path {
    Ray r;
    V tp, rad;
    uint32_t depth = 0;
    Rng rng;
    uint32_t medium = NONE;
    float density = 1.0f, prev_pdf = 0.0f, eta_scale = 1.0f;
    bool specular = true, alive = true;
};

static void add_rad(Path& p, const Cfg& c, V v, bool emission_or_background = false) {  // path_state.cuh:33-43
    bool indirect = p.depth > (emission_or_background ? 1u : 0u);
    if (indirect && c.clamp > 0.0f) {
        float m = (std::fabs(v.x) / 3.0f + std::fabs(v.y) / 3.0f + std::fabs(v.z) / 3.0f);
        if (m > c.clamp) v = mul(v, c.clamp / m);
    }
    acc(p.rad, v);
}

static float env_mix(const Scene& s) { return s.env.on && s.env.intensity > 0.0f ? 0.5f : 0.0f; }
static float diffuse_pdf(const Scene& s, V n, V d) {
    float pe = env_mix(s), pc = std::fmax(0.0f, dot(n, d)) * 0.31830988618f;
    return pe > 0.0f ? (1.0f - pe) * pc + pe * env_pdf(s.env, d) : pc;
}
static bool is_metal(const Mat& m) { return m.type == WF_MAT_METAL || (m.type == WF_MAT_DIFFUSE && m.metallic > 0.5f); }

// evaluateSurface(Cos) for the diffuse and metal models.
static V surface_cos(const Scene& s, const Mat& m, V n, V o, V i, float& pdf) {
    V f;
    if (is_metal(m)) {
        if (m.roughness <= 0.0f) { pdf = 0.0f; return V(); }
        f = ggx_eval(V(), m.albedo, m.roughness, n, o, i, pdf);
    } else {
        pdf = diffuse_pdf(s, n, i);
        f = mul(m.albedo, 0.31830988618f);
    }
    return mul(f, std::fmax(0.f, dot(n, i)));
}

static void nee_light(const PathCtx& x, Path& p, const Hit& h, V sn, const Mat& m) {  // sampleDirectLight
    const Scene& s = x.s;
    if (s.lights.empty()) return;
    uint32_t n = uint32_t(s.lights.size());
    uint32_t cand = std::min(uint32_t(p.rng.next() * n), n - 1);
    uint32_t li = p.rng.next() < s.lights[cand].alias_p ? cand : s.lights[cand].alias;
    const Light& L = s.lights[li];
    float ru = std::sqrt(p.rng.next()), v = p.rng.next();
    V lp = add(add(mul(L.a, 1.0f - ru), mul(L.b, ru * (1.0f - v))), mul(L.c, ru * v));
    V to = sub(lp, h.p);
    float d2 = len2(to), dist = std::sqrt(d2);
    V dir = divs(to, dist);
    float gc = std::fmax(0.0f, dot(h.gn, dir)), sc = std::fmax(0.0f, dot(sn, dir)), lc = std::fmax(0.0f, dot(L.n, neg(dir)));
    if (gc == 0.0f || sc == 0.0f || lc == 0.0f) return;
    V so = nudge(h.p, h.gn, dir, h.t), st = nudge(lp, L.n, neg(dir), dist);
    V seg = sub(st, so);
    float sd = len(seg);
    if (!(sd > T_MIN)) return;
    if (!s.ignore_occ && blocked(s, Ray{so, divs(seg, sd)}, sd - T_MIN)) return;
    float geo = lc * L.area / (d2 * L.pdf);
    float lpdf = L.pdf * d2 / (lc * L.area);
    float bpdf;
    V f = surface_cos(s, m, sn, neg(p.r.d), dir, bpdf);
    V direct = mul(had(f, s.mats[L.mat].emission), geo * mis(lpdf, bpdf));
    add_rad(p, x.c, had(p.tp, direct));
}

static void punctual_one(const PathCtx& x, Path& p, const Hit& h, V sn, const Mat& m, const Punct& L, float inv_pdf) {
    const Scene& s = x.s;
    V dir, inc;
    float dist = 1.0e30f;
    if (L.type == WF_LIGHT_DIRECTIONAL) {
        dir = neg(L.dir);
        inc = L.intensity;
    } else {
        V off = sub(L.pos, h.p);
        float d2 = len2(off);
        if (!(d2 > 0.0f)) return;
        dist = std::sqrt(d2);
        dir = divs(off, dist);
        float att = 1.0f / d2;
        if (L.range > 0.0f) {
            float ratio = dist / L.range;
            att *= std::fmax(0.0f, 1.0f - ratio * ratio * ratio * ratio);
        }
        if (L.type == WF_LIGHT_SPOT) {
            float c = dot(L.dir, neg(dir));
            float cone = std::fmin(1.0f, std::fmax(0.0f, (c - L.outer) / std::fmax(1.0e-6f, L.inner - L.outer)));
            att *= cone * cone;
        }
        inc = mul(L.intensity, att);
    }
    if (dot(sn, dir) <= 0.0f || dot(h.gn, dir) <= 0.0f || len2(inc) == 0.0f) return;
    Ray sh{nudge(h.p, h.gn, dir, h.t), dir};
    float sd = dist;
    if (L.type != WF_LIGHT_DIRECTIONAL) {
        V seg = sub(L.pos, sh.o);
        sd = len(seg);
        if (!(sd > T_MIN)) return;
        sh.d = divs(seg, sd);
    }
    if (!s.ignore_occ && blocked(s, sh, sd - T_MIN)) return;
    float ignored;
    V f = surface_cos(s, m, sn, neg(p.r.d), dir, ignored);
    add_rad(p, x.c, had(p.tp, mul(had(f, inc), inv_pdf)));
}

static void nee_punctual(const PathCtx& x, Path& p, const Hit& h, V sn, const Mat& m) {
    const Scene& s = x.s;
    for (uint32_t i = 0; i < s.directional; ++i) punctual_one(x, p, h, sn, m, s.punct[i], 1.0f);
    uint32_t n = uint32_t(s.punct.size()) - s.directional;
    if (n == 0) return;
    uint32_t i = s.directional + std::min(uint32_t(p.rng.next() * n), n - 1);
    punctual_one(x, p, h, sn, m, s.punct[i], float(n));
}

static void nee_env(const PathCtx& x, Path& p, const Hit& h, V sn, const Mat& m) {  // sampleDirectEnvironment
    const Scene& s = x.s;
    if (!s.env.on || s.env.intensity == 0.0f) return;
    EnvPick e = env_sample(s.env, p.rng);
    if (dot(sn, e.d) <= 0.0f || dot(h.gn, e.d) <= 0.0f || !(e.pdf > 0.0f)) return;
    if (!s.ignore_occ && blocked(s, Ray{nudge(h.p, h.gn, e.d, h.t), e.d}, 1.0e30f)) return;
    float bpdf;
    V f = surface_cos(s, m, sn, neg(p.r.d), e.d, bpdf);
    V direct = mul(had(f, env_lookup(s.env, e.d)), mis(e.pdf, bpdf) / e.pdf);
    add_rad(p, x.c, had(p.tp, direct));
}

static V gather(const PhotonMap* pm, const Hit& h, V sn, float radius);

// One shading event (shadePersistentPath, device_path_shading.cuh:175-319).
static void shade(const PathCtx& x, Path& p, bool did_hit, const Hit& h) {
    const Scene& s = x.s;
    const Cfg& c = x.c;
    if (c.debug) {
        V col = did_hit ? mul(add(h.n, mk(1, 1, 1)), 0.5f) : mk(0.05f, 0.10f, 0.25f);
        p.rad = col;
        p.alive = false;
        return;
    }
    if (!did_hit) {  // addEnvironmentOrSky
        if (s.env.on) {
            float w = p.depth > 0 && !p.specular ? mis(p.prev_pdf, env_pdf(s.env, p.r.d)) : 1.0f;
            add_rad(p, c, mul(had(p.tp, env_lookup(s.env, p.r.d)), w), true);
        } else if (!s.black) {
            float t = 0.5f * (p.r.d.y + 1.0f);
            V sky = add(mul(mk(1, 1, 1), 1.0f - t), mul(mk(0.5f, 0.7f, 1.0f), t));
            add_rad(p, c, had(p.tp, sky), true);
        }
        p.alive = false;
        return;
    }
    const Mat& m = s.mats[h.mat];
    if (p.medium != NONE) {  // Beer-Lambert through the enclosing dielectric
        const Mat& md = s.mats[p.medium];
        if (md.att_distance > 0.0f) {
            float dist = h.t * p.density;
            V sig = mk(-m_logf(std::fmax(md.att_color.x, 0.0001f)) / md.att_distance,
                       -m_logf(std::fmax(md.att_color.y, 0.0001f)) / md.att_distance,
                       -m_logf(std::fmax(md.att_color.z, 0.0001f)) / md.att_distance);
            p.tp = had(p.tp, mk(m_expf(-sig.x * dist), m_expf(-sig.y * dist), m_expf(-sig.z * dist)));
        }
    }
    if (m.type == WF_MAT_EMISSIVE) {
        float w = 1.0f;
        if (h.light != NONE) {
            const Light& L = s.lights[h.light];
            float lc = std::fmax(0.0f, dot(L.n, neg(p.r.d)));
            if (lc == 0.0f) w = 0.0f;
            else if (p.depth > 0 && !p.specular) w = mis(p.prev_pdf, L.pdf * h.t * h.t / (lc * L.area));
        }
        add_rad(p, c, mul(had(p.tp, m.emission), w), true);
        p.alive = false;
        return;
    }
    V sn = dot(h.n, h.gn) < 0.0f ? neg(h.n) : h.n;
    V dir;
    if (m.type == WF_MAT_DIELECTRIC) {  // continueDielectricSurface
        p.tp = had(p.tp, m.albedo);
        Boundary b = interface(unit(p.r.d), h.gn, sn, m.ior);
        float e2 = b.eta * b.eta;
        bool esc_r = false, esc_t = false;
        if (s.env.on && p.depth + 1 < c.depth) {
            if (b.R > 0.0f) {
                esc_r = !blocked(s, Ray{nudge(h.p, h.gn, b.refl, h.t), b.refl}, 1.0e30f);
                if (esc_r) add_rad(p, c, mul(had(p.tp, env_lookup(s.env, b.refl)), b.R));
            }
            if (b.R < 1.0f) {
                esc_t = !blocked(s, Ray{nudge(h.p, h.gn, b.trans, h.t), b.trans}, 1.0e30f);
                if (esc_t) add_rad(p, c, mul(had(p.tp, env_lookup(s.env, b.trans)), (1.0f - b.R) * e2));
            }
        }
        bool refl = b.R >= 1.0f || b.R > p.rng.next();
        if (!refl) {
            p.tp = mul(p.tp, e2);
            p.eta_scale /= e2;
            p.medium = b.front ? h.mat : NONE;
            p.density = b.front ? m.density * 1.0f : 1.0f;
        }
        if (refl ? esc_r : esc_t) p.alive = false;
        p.specular = true;
        p.prev_pdf = 0.0f;
        dir = refl ? b.refl : b.trans;
    } else if (is_metal(m) && !(m.roughness > 0.0f)) {  // mirror
        p.tp = had(p.tp, m.albedo);
        V refl = reflect(unit(p.r.d), sn);
        V jitter;
        for (;;) {  // randomInUnitSphere: three draws, rejection
            float a = 2.0f * p.rng.next() - 1.0f, b = 2.0f * p.rng.next() - 1.0f, cc = 2.0f * p.rng.next() - 1.0f;
            jitter = mk(a, b, cc);
            if (len2(jitter) < 1.0f) break;
        }
        dir = unit(add(refl, mul(jitter, m.roughness)));
        if (dot(dir, sn) <= 0.0f || dot(dir, h.gn) <= 0.0f) dir = reflect(unit(p.r.d), h.gn);
        p.specular = true;
        p.prev_pdf = 0.0f;
    } else {
        nee_light(x, p, h, sn, m);
        nee_punctual(x, p, h, sn, m);
        nee_env(x, p, h, sn, m);
        if (!is_metal(m)) {
            if (x.pm) add_rad(p, c, had(p.tp, had(m.albedo, gather(x.pm, h, sn, c.gather))));
            float pe = env_mix(s);
            dir = pe > 0.0f && p.rng.next() < pe ? env_sample(s.env, p.rng).d : cos_hemi(sn, p.rng);
            float cs = dot(sn, dir), pdf = diffuse_pdf(s, sn, dir);
            if (!(pdf > 0.0f) || cs <= 0.0f || dot(dir, h.gn) <= 0.0f) {
                p.alive = false;
            } else {
                p.tp = mul(had(p.tp, m.albedo), cs * 0.31830988618f / pdf);
                p.prev_pdf = pdf;
                p.specular = false;
            }
        } else {  // continueGlossySurface
            V o = neg(p.r.d);
            float ch = p.rng.next(), u = p.rng.next(), v = p.rng.next();
            dir = ggx_sample(V(), m.albedo, m.roughness, sn, o, ch, u, v);
            float pdf;
            V f = ggx_eval(V(), m.albedo, m.roughness, sn, o, dir, pdf);
            if (!(pdf > 0.0f) || dot(dir, h.gn) <= 0.0f) {
                p.alive = false;
            } else {
                p.tp = mul(had(p.tp, f), std::fmax(0.0f, dot(sn, dir)) / pdf);
                p.prev_pdf = pdf;
                p.specular = false;
            }
        }
    }
    if (!p.alive) return;
    p.r.o = nudge(h.p, h.gn, dir, h.t);
    p.r.d = dir;
    ++p.depth;
    if (p.depth >= c.depth) { p.alive = false; return; }
    if (p.depth >= c.rr) {
        float q = std::fmin(0.95f, std::fmax(0.05f, p.eta_scale * std::fmax(p.tp.x, std::fmax(p.tp.y, p.tp.z))));
        if (p.rng.next() > q) { p.alive = false; return; }
        p.tp = mul(p.tp, 1.0f / q);
    }
}

// ------------------------------------------------------------ photon map
struct Photon {
    V pos, dir, flux;
    Rng rng;
    uint32_t bounces = 0, channel = 3;
    bool valid = false;
};
struct PhotonMap {
    std::vector<Photon> ph;
    std::vector<std::vector<uint32_t>> cells;  // each list in descending photon index
    uint32_t res;
    V lo, hi;
    uint32_t stored = 0;
};

static PhotonMap* build_photons(const Scene& s, const wf_render_config* c) {  // photon_mapping.cu:4-89
    auto pm = std::make_unique<PhotonMap>();
    uint32_t n = c->photon_count;
    pm->ph.resize(n);
    if (s.lights.empty()) return pm.release();
    uint32_t nl = uint32_t(s.lights.size());
    for (uint32_t i = 0; i < n; ++i) {
        Photon& P = pm->ph[i];
        P.rng = seed_rng(photon_key(i, c->photon_seed, c->rng), c->rng);
        uint32_t cand = std::min(uint32_t(P.rng.next() * nl), nl - 1);
        uint32_t li = P.rng.next() < s.lights[cand].alias_p ? cand : s.lights[cand].alias;
        const Light& L = s.lights[li];
        float ru = std::sqrt(P.rng.next()), v = P.rng.next();
        V pt = add(mul(L.a, 1.0f - ru), mul(add(mul(L.b, 1.0f - v), mul(L.c, v)), ru));
        P.dir = cos_hemi(L.n, P.rng);
        const Mat& m = s.mats[L.mat];
        P.flux = mul(m.emission, L.area * 3.14159265359f / float(n));
        if (c->spectral) {
            P.channel = std::min(uint32_t(P.rng.next() * 3.0f), 2u);
            float e = P.channel == 0 ? m.emission.x : P.channel == 1 ? m.emission.y : m.emission.z;
            float cf = e * (L.area * 3.14159265359f * 3.0f / float(n));
            P.flux = V();
            if (P.channel == 0) P.flux.x = cf; else if (P.channel == 1) P.flux.y = cf; else P.flux.z = cf;
        }
        P.pos = add(pt, mul(L.n, 0.001f));
    }
    std::vector<std::thread> pool;
    std::atomic<uint32_t> next{0};
    unsigned T = std::max(1u, std::thread::hardware_concurrency());
    for (unsigned t = 0; t < T; ++t)
        pool.emplace_back([&] {
            for (;;) {
                uint32_t i = next.fetch_add(1);
                if (i >= n) break;
                Photon P = pm->ph[i];
                Ray r{P.pos, P.dir};
                for (uint32_t d = 0; d < c->photon_max_depth; ++d) {
                    Best b = closest(s, r);
                    Hit h;
                    if (!finish(s, r, b, h)) break;
                    if (h.mat >= s.mats.size()) break;
                    const Mat& m = s.mats[h.mat];
                    V nrm = dot(h.n, neg(r.d)) >= 0.0f ? h.n : neg(h.n);
                    if (m.type == WF_MAT_DIFFUSE) {
                        if (P.bounces == 0) break;
                        P.pos = h.p;
                        P.dir = neg(r.d);
                        P.valid = true;
                        pm->ph[i] = P;
                        break;
                    }
                    V dir;
                    if (m.type == WF_MAT_METAL) {
                        dir = unit(reflect(unit(r.d), nrm));
                    } else if (m.type == WF_MAT_DIELECTRIC) {
                        float ior = m.ior;
                        if (m.dispersion > 0.0f && P.channel < 3) ior += (float(P.channel) - 1.0f) * m.dispersion;
                        Boundary bd = interface(unit(r.d), h.gn, h.n, ior);
                        bool refl = bd.R >= 1.0f || bd.R > P.rng.next();
                        dir = refl ? bd.refl : bd.trans;
                    } else {
                        dir = cos_hemi(nrm, P.rng);
                    }
                    if (m.type == WF_MAT_METAL || m.type == WF_MAT_DIELECTRIC) ++P.bounces;
                    P.flux = had(P.flux, m.albedo);
                    r = Ray{nudge(h.p, h.gn, dir, h.t), dir};
                }
            }
        });
    for (auto& t : pool) t.join();
    pm->res = c->photon_grid_resolution;
    pm->lo = mk3(c->photon_grid_min);
    pm->hi = mk3(c->photon_grid_max);
    if (pm->lo.x == pm->hi.x && pm->lo.y == pm->hi.y && pm->lo.z == pm->hi.z) {  // bounds of the stored photons
        V lo = mk(INFINITY, INFINITY, INFINITY), hi = mk(-INFINITY, -INFINITY, -INFINITY);
        bool any = false;
        for (const Photon& P : pm->ph)
            if (P.valid) {
                any = true;
                lo = mk(std::fmin(lo.x, P.pos.x), std::fmin(lo.y, P.pos.y), std::fmin(lo.z, P.pos.z));
                hi = mk(std::fmax(hi.x, P.pos.x), std::fmax(hi.y, P.pos.y), std::fmax(hi.z, P.pos.z));
            }
        if (!any) { lo = mk(-1, -1, -1); hi = mk(1, 1, 1); }
        if (!(hi.x > lo.x)) hi.x = lo.x + 1.0f;
        if (!(hi.y > lo.y)) hi.y = lo.y + 1.0f;
        if (!(hi.z > lo.z)) hi.z = lo.z + 1.0f;
        pm->lo = lo;
        pm->hi = hi;
    }
    pm->cells.assign(size_t(pm->res) * pm->res * pm->res, {});
    V ext = sub(pm->hi, pm->lo);
    int R = int(pm->res);
    for (uint32_t i = n; i-- > 0;) {  // descending index = the order serial head insertion leaves
        const Photon& P = pm->ph[i];
        if (!P.valid) continue;
        V off = sub(P.pos, pm->lo);
        V nn = mk(off.x / ext.x, off.y / ext.y, off.z / ext.z);
        int x = std::min(std::max(int(nn.x * pm->res), 0), R - 1);
        int y = std::min(std::max(int(nn.y * pm->res), 0), R - 1);
        int z = std::min(std::max(int(nn.z * pm->res), 0), R - 1);
        if (nn.x < 0.0f || nn.y < 0.0f || nn.z < 0.0f || nn.x > 1.0f || nn.y > 1.0f || nn.z > 1.0f) continue;
        pm->cells[(size_t(z) * pm->res + y) * pm->res + x].push_back(i);
    }
    for (const Photon& P : pm->ph) pm->stored += P.valid ? 1 : 0;
    return pm.release();
}

static V gather(const PhotonMap* pm, const Hit& h, V sn, float radius) {  // photon_mapping.cu:91-163
    V ext = sub(pm->hi, pm->lo);
    V off = sub(h.p, pm->lo);
    V nn = mk(off.x / ext.x, off.y / ext.y, off.z / ext.z);
    int R = int(pm->res);
    int cx = std::min(std::max(int(nn.x * pm->res), 0), R - 1);
    int cy = std::min(std::max(int(nn.y * pm->res), 0), R - 1);
    int cz = std::min(std::max(int(nn.z * pm->res), 0), R - 1);
    float sr = std::fmax(radius * 4.0f, 0.1f);
    int cr = std::max(1, int(std::ceil(sr * pm->res / std::fmax(ext.x, 0.0001f))));
    float sr2 = sr * sr;
    float dist[64];
    uint32_t idx[64];
    uint32_t count = 0, far = 0;
    float far2 = 0.0f;
    for (uint32_t i = 0; i < 64; ++i) { dist[i] = 0.0f; idx[i] = NONE; }
    for (int z = cz - cr; z <= cz + cr; ++z)
        for (int y = cy - cr; y <= cy + cr; ++y)
            for (int x = cx - cr; x <= cx + cr; ++x) {
                if (x < 0 || y < 0 || z < 0 || x >= R || y >= R || z >= R) continue;
                for (uint32_t i : pm->cells[(size_t(z) * pm->res + y) * pm->res + x]) {
                    const Photon& P = pm->ph[i];
                    V po = sub(P.pos, h.p);
                    float d2 = dot(po, po), cs = dot(sn, P.dir);
                    if (d2 > sr2 || cs <= 0.0f) continue;
                    if (count < 64) {
                        dist[count] = d2;
                        idx[count] = i;
                        if (d2 > far2) { far2 = d2; far = count; }
                        ++count;
                    } else if (d2 < far2) {
                        dist[far] = d2;
                        idx[far] = i;
                        far = 0;
                        far2 = dist[0];
                        for (uint32_t k = 1; k < 64; ++k)
                            if (dist[k] > far2) { far2 = dist[k]; far = k; }
                    }
                }
            }
    if (count == 0) return V();
    float g2 = sr2;
    if (count >= 16) {
        g2 = 0.0f;
        for (uint32_t k = 0; k < count; ++k) g2 = std::fmax(g2, dist[k]);
        g2 = std::fmax(g2, radius * radius);
    }
    float g = std::sqrt(g2);
    V out;
    for (uint32_t k = 0; k < count; ++k) {
        const Photon& P = pm->ph[idx[k]];
        float w = std::fmax(0.0f, 1.0f - std::sqrt(dist[k]) / g);
        acc(out, mul(P.flux, w * dot(sn, P.dir)));
    }
    return mul(out, 3.0f / (3.14159265359f * g2));
}

struct Handle {
    std::unique_ptr<Scene> scene;
    std::unique_ptr<PhotonMap> photons;
    std::string key;
};

// ------------------------------------------------- FP64 adjoint (test only)
// Double-precision restatement of the differentiable renderer of
// wavefront-path-tracer_b200/csrc/wf_adjoint.cu (Oren-Nayar BRDF per
// triangle, triangle-light next events, cosine continuations).  Every
// geometric decision (ray directions, hits, shadow rays, RNG draws) is made
// in float exactly as on the GPU, so both follow the same paths; BRDF
// values, path weights, terms and gradients are carried in double.
struct OrenNayarD {
    double value, d_sigma;
};
static OrenNayarD oren_nayar_d(V n, V wo, V wi, double sigma) {
    double nx = n.x, ny = n.y, nz = n.z;
    double ci = std::min(1.0, std::max(0.0, nx * wi.x + ny * wi.y + nz * wi.z));
    double co = std::min(1.0, std::max(0.0, nx * wo.x + ny * wo.y + nz * wo.z));
    double si = std::sqrt(std::max(0.0, 1.0 - ci * ci)), so = std::sqrt(std::max(0.0, 1.0 - co * co));
    double g = 0.0;
    if (si > 1e-4 && so > 1e-4) {
        double tix = (wi.x - nx * ci) / si, tiy = (wi.y - ny * ci) / si, tiz = (wi.z - nz * ci) / si;
        double tox = (wo.x - nx * co) / so, toy = (wo.y - ny * co) / so, toz = (wo.z - nz * co) / so;
        double cphi = std::max(0.0, tix * tox + tiy * toy + tiz * toz);
        double sin_alpha = ci < co ? si : so;
        double tan_beta = ci < co ? so / std::max(co, 1e-4) : si / std::max(ci, 1e-4);
        g = cphi * sin_alpha * tan_beta;
    }
    double s2 = sigma * sigma;
    double a = 1.0 - 0.5 * s2 / (s2 + 0.33), b = 0.45 * s2 / (s2 + 0.09);
    double da = -0.33 * sigma / ((s2 + 0.33) * (s2 + 0.33)), db = 0.081 * sigma / ((s2 + 0.09) * (s2 + 0.09));
    return OrenNayarD{a + b * g, da + db * g};
}

struct D3 {
    double x = 0, y = 0, z = 0;
};
static D3 d3(V v) { return D3{v.x, v.y, v.z}; }
static D3 dmul(D3 a, D3 b) { return D3{a.x * b.x, a.y * b.y, a.z * b.z}; }
static D3 dscale(D3 a, double s) { return D3{a.x * s, a.y * s, a.z * s}; }
static D3 dadd(D3 a, D3 b) { return D3{a.x + b.x, a.y + b.y, a.z + b.z}; }
static D3 dsub(D3 a, D3 b) { return D3{a.x - b.x, a.y - b.y, a.z - b.z}; }
static double ddot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

struct DiffCtx {
    const Scene& s;
    const wf_diff_config& c;
    V cam_p, cam_f, cam_r, cam_u;
    float aspect, tan_half;
    const float* albedo;
    const float* rough;
};

// kAdjoint = false: returns U (path radiance at emission scale 1).
// kAdjoint = true: adds delta . dU/dtheta into ga/gr and returns U.
template <bool kAdjoint>
static D3 diff_path_d(const DiffCtx& x, uint32_t px, uint32_t py, uint32_t sample, D3 total, D3 delta, double* ga,
                      double* gr, bool& bad) {
    const Scene& s = x.s;
    uint32_t pixel = py * x.c.width + px;
    Rng rng = seed_rng(pixel_key(pixel, sample, x.c.rng), x.c.rng);
    float u = (float(px) + rng.next()) / float(x.c.width);
    float v = (float(py) + rng.next()) / float(x.c.height);
    float cx = (2.0f * u - 1.0f) * x.aspect * x.tan_half;
    float cy = (1.0f - 2.0f * v) * x.tan_half;
    Ray r{x.cam_p, unit(add(add(x.cam_f, mul(x.cam_r, cx)), mul(x.cam_u, cy)))};
    D3 beta{1, 1, 1}, sum;
    for (uint32_t depth = 0; depth < x.c.max_depth; ++depth) {
        Best b = closest(s, r);
        Hit h;
        if (!finish(s, r, b, h)) break;
        const Mat& m = s.mats[h.mat];
        if (m.type == WF_MAT_EMISSIVE) {
            if (depth == 0) sum = dadd(sum, dmul(beta, d3(m.emission)));
            break;
        }
        if (b.kind == WF_HIT_SPHERE) break;
        uint32_t k = b.prim;
        if (k >= x.c.parameter_count) {
            bad = true;
            break;
        }
        D3 albedo{x.albedo[3 * k], x.albedo[3 * k + 1], x.albedo[3 * k + 2]};
        double sigma = x.rough[k];
        V gn = h.gn, n = h.n;
        if (dot(n, gn) < 0.0f) n = neg(n);
        V wo = neg(r.d);
        D3 nee_free;
        double nee_dsigma = 0.0;
        if (!s.lights.empty()) {
            uint32_t nl = uint32_t(s.lights.size());
            uint32_t cand = std::min(uint32_t(rng.next() * nl), nl - 1);
            uint32_t li = rng.next() < s.lights[cand].alias_p ? cand : s.lights[cand].alias;
            const Light& L = s.lights[li];
            float ru = std::sqrt(rng.next()), lv = rng.next();
            V lp = add(add(mul(L.a, 1.0f - ru), mul(L.b, ru * (1.0f - lv))), mul(L.c, ru * lv));
            V to = sub(lp, h.p);
            float d2 = len2(to), dist = std::sqrt(d2);
            V wl = divs(to, dist);
            float cg = dot(gn, wl), cs = dot(n, wl), cl = dot(L.n, neg(wl));
            if (cg > 0.0f && cs > 0.0f && cl > 0.0f) {
                V so = nudge(h.p, gn, wl, h.t), st = nudge(lp, L.n, neg(wl), dist);
                V seg = sub(st, so);
                float sd = len(seg);
                if (sd > T_MIN && !blocked(s, Ray{so, divs(seg, sd)}, sd - T_MIN)) {
                    OrenNayarD on = oren_nayar_d(n, wo, wl, sigma);
                    double geo = double(cl) * L.area / (double(d2) * L.pdf);
                    nee_free = dscale(dmul(beta, d3(s.mats[L.mat].emission)), on.value / M_PI * double(cs) * geo);
                    nee_dsigma = on.value > 0.0 ? on.d_sigma / on.value : 0.0;
                    sum = dadd(sum, dmul(albedo, nee_free));
                }
            }
        }
        float u1 = rng.next(), u2 = rng.next();
        float rad = std::sqrt(u1), phi = 6.28318530718f * u2;
        float sx = rad * m_cosf(phi), sy = rad * m_sinf(phi), sz = std::sqrt(1.0f - u1);
        V helper = std::fabs(n.x) > 0.1f ? mk(0, 1, 0) : mk(1, 0, 0);
        V t = unit(cross(helper, n));
        V bt = cross(n, t);
        V wi = unit(add(add(mul(t, sx), mul(bt, sy)), mul(n, sz)));
        bool continues = depth + 1 < x.c.max_depth && dot(wi, gn) > 0.0f;
        OrenNayarD on = continues ? oren_nayar_d(n, wo, wi, sigma) : OrenNayarD{0, 0};
        if (kAdjoint) {
            D3 after = dsub(total, sum);
            D3 g;
            double gs = 0.0;
            if (continues) {
                g = D3{albedo.x > 0 ? after.x / albedo.x : 0, albedo.y > 0 ? after.y / albedo.y : 0,
                       albedo.z > 0 ? after.z / albedo.z : 0};
                gs = on.value > 0 ? ddot(delta, after) * (on.d_sigma / on.value) : 0.0;
            }
            g = dadd(g, nee_free);
            gs += ddot(delta, dmul(albedo, nee_free)) * nee_dsigma;
            ga[3 * k] += delta.x * g.x;
            ga[3 * k + 1] += delta.y * g.y;
            ga[3 * k + 2] += delta.z * g.z;
            gr[k] += gs;
        }
        if (!continues) break;
        beta = dmul(beta, dscale(albedo, on.value));
        r = Ray{nudge(h.p, gn, wi, h.t), wi};
    }
    return sum;
}

}  // namespace port

using namespace port;

extern "C" {

void* oracle_scene_create(const wf_scene_desc* d, const wf_environment* env) {
    Scene* s = build_scene(d, env);
    if (!s) return nullptr;
    Handle* h = new Handle;
    h->scene.reset(s);
    return h;
}

void oracle_scene_destroy(void* h) { delete static_cast<Handle*>(h); }

uint32_t oracle_light_count(void* h) { return uint32_t(static_cast<Handle*>(h)->scene->lights.size()); }

void oracle_trace(void* handle, const wf_ray* rays, uint32_t n, wf_hit* out) {
    const Scene& s = *static_cast<Handle*>(handle)->scene;
    for (uint32_t i = 0; i < n; ++i) {
        Ray r{mk3(rays[i].origin), mk3(rays[i].direction)};
        Best b = closest(s, r);
        Hit h;
        wf_hit& o = out[i];
        std::memset(&o, 0, sizeof(o));
        o.instance = NONE;
        o.primitive = NONE;
        if (!finish(s, r, b, h)) {
            o.t = 1e30f;
            o.material = NONE;
            o.light_index = NONE;
            continue;
        }
        o.t = h.t;
        o.position[0] = h.p.x; o.position[1] = h.p.y; o.position[2] = h.p.z;
        o.geometric_normal[0] = h.gn.x; o.geometric_normal[1] = h.gn.y; o.geometric_normal[2] = h.gn.z;
        o.normal[0] = h.n.x; o.normal[1] = h.n.y; o.normal[2] = h.n.z;
        o.material = h.mat;
        o.light_index = h.light;
        o.kind = b.kind;
        o.primitive = b.prim;
        o.instance = b.kind == WF_HIT_MESH ? b.inst : NONE;
        if (b.kind != WF_HIT_SPHERE) { o.u = b.u; o.v = b.v; }
    }
}

void oracle_occluded(void* handle, const wf_ray* rays, const float* limit, uint32_t n, uint8_t* out) {
    const Scene& s = *static_cast<Handle*>(handle)->scene;
    for (uint32_t i = 0; i < n; ++i) out[i] = blocked(s, Ray{mk3(rays[i].origin), mk3(rays[i].direction)}, limit[i]) ? 1 : 0;
}

uint32_t oracle_photons(void* handle, const wf_render_config* c, float* records) {
    Handle* h = static_cast<Handle*>(handle);
    std::unique_ptr<PhotonMap> pm(build_photons(*h->scene, c));
    for (uint32_t i = 0; i < c->photon_count; ++i) {
        const Photon& P = pm->ph[i];
        float* o = records + 8 * size_t(i);
        o[0] = P.pos.x; o[1] = P.pos.y; o[2] = P.pos.z;
        o[3] = P.dir.x; o[4] = P.dir.y; o[5] = P.dir.z;
        o[6] = P.flux.x + P.flux.y + P.flux.z;
        o[7] = P.valid ? 1.0f : 0.0f;
    }
    return pm->stored;
}

// Renders absolute samples [start, start + count) of a tile one path at a
// time on `threads` host threads.  fb: FP32 sums, accumulated per pixel in
// sample order; counts: per-sample, per-bounce number of live paths.
int oracle_render(void* handle, const wf_camera* cam, const wf_render_config* c, uint32_t x0, uint32_t y0, uint32_t tw,
                  uint32_t th, uint32_t start, uint32_t count, float* fb, uint32_t* counts, int threads) {
    Handle* h = static_cast<Handle*>(handle);
    const Scene& s = *h->scene;
    Cfg cfg;
    cfg.width = c->width;
    cfg.height = c->height;
    cfg.depth = c->max_depth;
    cfg.rr = c->rr_start_depth;
    cfg.rng = c->rng;
    cfg.debug = c->debug;
    cfg.clamp = c->indirect_clamp;
    cfg.gather = c->gather_radius;
    cfg.cam_p = mk3(cam->position);
    cfg.cam_f = mk3(cam->forward);
    cfg.cam_r = mk3(cam->right);
    cfg.cam_u = mk3(cam->up);
    cfg.aspect = cam->aspect_ratio;
    cfg.tan_half = m_tanf(cam->vertical_fov * 0.5f);
    const PhotonMap* pm = nullptr;
    if (c->caustics && c->photon_count) {
        char key[96];
        std::snprintf(key, sizeof(key), "%u/%u/%u/%u/%u", c->photon_count, c->photon_seed, c->photon_max_depth,
                      c->photon_grid_resolution, c->rng);
        if (!h->photons || h->key != key) {
            h->photons.reset(build_photons(s, c));
            h->key = key;
        }
        if (c->caustic_gather) pm = h->photons.get();
    }
    PathCtx ctx{s, cfg, pm};
    uint32_t pixels = tw * th;
    std::vector<std::atomic<uint32_t>> live(size_t(count) * cfg.depth);
    for (auto& a : live) a = 0;
    if (threads <= 0) threads = int(std::max(1u, std::thread::hardware_concurrency()));
    std::atomic<uint32_t> next{0};
    // Each pixel accumulates its samples in sample order, as the reference's
    // framebuffer does (one path per pixel per sample pass).
    std::vector<float> acc_fb(size_t(pixels) * 3, 0.0f);
    auto work_fb = [&] {
        for (;;) {
            uint32_t lp = next.fetch_add(1);
            if (lp >= pixels) break;
            uint32_t x = x0 + lp % tw, y = y0 + lp / tw;
            uint32_t pixel = y * cfg.width + x;
            float* f = &acc_fb[3 * size_t(lp)];
            for (uint32_t k = 0; k < count; ++k) {
                Path p;
                p.rng = seed_rng(pixel_key(pixel, start + k, cfg.rng), cfg.rng);
                float u = (float(x) + p.rng.next()) / float(cfg.width);
                float v = (float(y) + p.rng.next()) / float(cfg.height);
                float cx = (2.0f * u - 1.0f) * cfg.aspect * cfg.tan_half;
                float cy = (1.0f - 2.0f * v) * cfg.tan_half;
                p.r = Ray{cfg.cam_p, unit(add(add(cfg.cam_f, mul(cfg.cam_r, cx)), mul(cfg.cam_u, cy)))};
                p.tp = mk(1, 1, 1);
                for (uint32_t b = 0; b < cfg.depth && p.alive; ++b) {
                    live[size_t(k) * cfg.depth + b].fetch_add(1);
                    Best best = closest(s, p.r);
                    Hit hit;
                    bool did = finish(s, p.r, best, hit);
                    shade(ctx, p, did, hit);
                }
                f[0] += p.rad.x;
                f[1] += p.rad.y;
                f[2] += p.rad.z;
            }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) pool.emplace_back(work_fb);
    for (auto& t : pool) t.join();
    std::memcpy(fb, acc_fb.data(), sizeof(float) * acc_fb.size());
    if (counts)
        for (size_t i = 0; i < live.size(); ++i) counts[i] = live[i].load();
    return 0;
}


// FP64 forward and adjoint of the differentiable renderer over the config's
// crop.  image (optional): crop_height x crop_width x 3 doubles.  d_image
// (optional, full width x height x 3 floats): dLoss/dImage; gradients are
// ADDED to d_albedo (3 per parameter), d_roughness, d_scale.
int oracle_diff(void* handle, const wf_camera* cam, const wf_diff_config* c, const float* albedo,
                const float* roughness, double emission_scale, const float* d_image, double* image, double* d_albedo,
                double* d_roughness, double* d_scale, int threads) {
    Handle* hd = static_cast<Handle*>(handle);
    DiffCtx x{*hd->scene, *c, mk3(cam->position), mk3(cam->forward), mk3(cam->right), mk3(cam->up),
              cam->aspect_ratio, m_tanf(cam->vertical_fov * 0.5f), albedo, roughness};
    uint32_t cw = c->crop_width ? c->crop_width : c->width, ch = c->crop_height ? c->crop_height : c->height;
    uint32_t pixels = cw * ch, np = c->parameter_count;
    if (threads <= 0) threads = int(std::max(1u, std::thread::hardware_concurrency()));
    std::vector<std::vector<double>> ga(threads), gr(threads);
    std::vector<double> gs(threads, 0.0);
    std::atomic<uint32_t> next{0};
    std::atomic<bool> bad{false};
    auto work = [&](int w) {
        if (d_image) {
            ga[w].assign(size_t(np) * 3, 0.0);
            gr[w].assign(np, 0.0);
        }
        for (;;) {
            uint32_t i = next.fetch_add(1);
            if (i >= pixels) break;
            uint32_t px = c->crop_x + i % cw, py = c->crop_y + i / cw;
            D3 acc;
            D3 delta, gpix;
            if (d_image) {
                const float* g = d_image + 3 * (size_t(py) * c->width + px);
                gpix = D3{g[0], g[1], g[2]};
                delta = dscale(gpix, emission_scale / double(c->spp));
            }
            bool b = false;
            for (uint32_t k = 0; k < c->spp; ++k) {
                uint32_t sample = c->sample_start + k;
                D3 total = diff_path_d<false>(x, px, py, sample, D3{}, D3{}, nullptr, nullptr, b);
                acc = dadd(acc, total);
                if (d_image) {
                    diff_path_d<true>(x, px, py, sample, total, delta, ga[w].data(), gr[w].data(), b);
                    gs[w] += ddot(gpix, total) / double(c->spp);
                }
            }
            if (b) bad = true;
            if (image) {
                double* o = image + 3 * size_t(i);
                double sc = emission_scale / double(c->spp);
                o[0] = acc.x * sc;
                o[1] = acc.y * sc;
                o[2] = acc.z * sc;
            }
        }
    };
    std::vector<std::thread> pool;
    for (int w = 0; w < threads; ++w) pool.emplace_back(work, w);
    for (auto& t : pool) t.join();
    if (d_image) {
        for (int w = 0; w < threads; ++w) {
            for (size_t j = 0; j < size_t(np) * 3; ++j) d_albedo[j] += ga[w][j];
            for (size_t j = 0; j < np; ++j) d_roughness[j] += gr[w][j];
            *d_scale += gs[w];
        }
    }
    return bad ? 1 : 0;
}

}  // extern "C"
