// scenes.cpp — the procedural scene generators (seeded stand-ins for the reference's .glb
// scenes), the camera basis and the light luminance prefix sums, and the flat phx_scene view of a
// generated scene.  Host-only C++ with no CUDA dependency, so the CPU oracle library compiles the
// same file and a CPU-only caller can generate a scene without loading the CUDA library.
#include "host.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace phx {

namespace {
constexpr float INF = 1e9f;
constexpr float PI = 3.141592654f;
inline float u2f(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
} // namespace

void SceneStore::view(phx_scene *s) const {
    std::memset(s, 0, sizeof(*s));
    s->triangles = tris.data();
    s->n_triangles = (uint32_t)tris.size();
    s->emissive_triangles = etris.empty() ? nullptr : etris.data();
    s->n_emissive_triangles = (uint32_t)etris.size();
    s->materials = mats.data();
    s->uv_transforms = uvs.data();
    s->n_materials = (uint32_t)mats.size();
    s->lights = lights.empty() ? nullptr : lights.data();
    s->n_lights = (uint32_t)lights.size();
    s->lum_pref_sum = lum.empty() ? nullptr : lum.data();
    s->tex_meta = tex_meta.empty() ? nullptr : tex_meta.data();
    s->n_textures = (uint32_t)tex_meta.size();
    s->tex_atlas = atlas.empty() ? nullptr : atlas.data();
    s->tex_atlas_bytes = atlas.size();
    s->envmap = envmap.empty() ? nullptr : envmap.data();
    s->envmap_width = env_w;
    s->envmap_height = env_h;
    s->camera = camera;
}

// ---- procedural scenes --------------------------------------------------------------------------
namespace {

struct V3 {
    double x, y, z;
};
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 vcross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double vdot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 vnorm(V3 a) {
    double l = std::sqrt(vdot(a, a));
    return l > 0 ? a * (1.0 / l) : a;
}

struct Pcg { // the renderer's PCG stream (random.h:16-36) drives every generator choice
    uint32_t s;
    explicit Pcg(uint32_t seed) {
        s = 2891336453u + seed;
        s = s * 747796405u + 2891336453u;
    }
    uint32_t next() {
        uint32_t old = s;
        s = s * 747796405u + 2891336453u;
        return ((old >> ((old >> 28u) + 4u)) ^ old) * 277803737u;
    }
    double uni() { return (double)next() / 4294967296.0; }
    double uni(double a, double b) { return a + (b - a) * uni(); }
};

phx_f4 F4(V3 v) { return {(float)v.x, (float)v.y, (float)v.z, 0.0f}; }

phx_material make_material(float r, float g, float b, float metallic, float roughness) {
    // make_default_material (src/parsers/material.cpp:9-30) with the given factors
    phx_material m{};
    m.base_color = {r, g, b, 1.0f};
    m.emissive = {0.0f, 0.0f, 0.0f, 0.0f};
    m.att_color = {1.0f, 1.0f, 1.0f, 0.0f};
    m.metallic = metallic;
    m.roughness = roughness;
    m.transmission = 0.0f;
    m.ior = 1.5f;
    m.att_dist = INF;
    m.thickness = 0.0f;
    m.diff_index = m.emis_index = m.norm_index = m.occlusion_index = m.metal_rough_index = m.transmission_index =
        PHX_NO_TEXTURE;
    return m;
}

phx_uv_transform_block identity_uv() {
    phx_uv_transform id{};
    id.uv_offset = {0.0f, 0.0f};
    id.uv_scale = {1.0f, 1.0f};
    id.uv_rotation = 0.0f;
    phx_uv_transform_block b{};
    b.diff = b.emis = b.norm = b.occlusion = b.metal_rough = b.transmission = id;
    return b;
}

struct Gen {
    SceneStore &s;
    explicit Gen(SceneStore &st) : s(st) {}

    uint32_t material(const phx_material &m) {
        s.mats.push_back(m);
        s.uvs.push_back(identity_uv());
        return (uint32_t)s.mats.size() - 1;
    }

    // one triangle with per-vertex normals; tangent as parse_mesh computes it without UVs
    // (scene.cpp:83-95: det = 0 -> (1,0,0))
    void tri(V3 p0, V3 p1, V3 p2, V3 n0, V3 n1, V3 n2, uint32_t mat) {
        phx_triangle t{};
        t.v0 = F4(p0);
        t.v1 = F4(p1);
        t.v2 = F4(p2);
        t.n0 = F4(vnorm(n0));
        t.n1 = F4(vnorm(n1));
        t.n2 = F4(vnorm(n2));
        t.t0 = t.t1 = t.t2 = {1.0f, 0.0f, 0.0f, 0.0f};
        t.uv0 = t.uv1 = t.uv2 = {0.0f, 0.0f};
        t.mat_index = mat;
        s.tris.push_back(t);
    }
    void flat_tri(V3 p0, V3 p1, V3 p2, V3 n, uint32_t mat) { tri(p0, p1, p2, n, n, n, mat); }
    // quad a-b-c-d (counter-clockwise seen from the normal side)
    void quad(V3 a, V3 b, V3 c, V3 d, V3 n, uint32_t mat) {
        flat_tri(a, b, c, n, mat);
        flat_tri(a, c, d, n, mat);
    }
    // emissive mesh -> LIGHT_TEXTURED (scene.cpp:115-130): power = pi * emissive * area
    void emissive_quad(V3 a, V3 b, V3 c, V3 d, V3 n, uint32_t mat, V3 emissive) {
        uint32_t start_tri = (uint32_t)s.tris.size();
        quad(a, b, c, d, n, mat);
        uint32_t estart = (uint32_t)s.etris.size();
        float area = 0.0f;
        for (uint32_t j = start_tri; j < (uint32_t)s.tris.size(); j++) {
            const phx_triangle &t = s.tris[j];
            s.etris.push_back(t);
            float e1[3] = {t.v1.x - t.v0.x, t.v1.y - t.v0.y, t.v1.z - t.v0.z};
            float e2[3] = {t.v2.x - t.v0.x, t.v2.y - t.v0.y, t.v2.z - t.v0.z};
            float cx = e1[1] * e2[2] - e1[2] * e2[1], cy = e1[2] * e2[0] - e1[0] * e2[2],
                  cz = e1[0] * e2[1] - e1[1] * e2[0];
            area += 0.5f * std::sqrt(cx * cx + cy * cy + cz * cz);
        }
        phx_light l{};
        l.kind = PHX_LIGHT_TEXTURED;
        l.power = {PI * (float)emissive.x * area, PI * (float)emissive.y * area, PI * (float)emissive.z * area, 0.0f};
        l.aux = {u2f(PHX_NO_TEXTURE), u2f(estart), u2f((uint32_t)s.tris.size() - start_tri), area};
        s.lights.push_back(l);
    }
    void box(V3 lo, V3 hi, double yaw, uint32_t mat) {
        V3 c = (lo + hi) * 0.5, h = (hi - lo) * 0.5;
        double cs = std::cos(yaw), sn = std::sin(yaw);
        auto P = [&](double sx, double sy, double sz) {
            double x = sx * h.x, z = sz * h.z;
            return V3{c.x + cs * x - sn * z, c.y + sy * h.y, c.z + sn * x + cs * z};
        };
        auto N = [&](double x, double y, double z) { return V3{cs * x - sn * z, y, sn * x + cs * z}; };
        quad(P(-1, -1, 1), P(1, -1, 1), P(1, 1, 1), P(-1, 1, 1), N(0, 0, 1), mat);
        quad(P(1, -1, -1), P(-1, -1, -1), P(-1, 1, -1), P(1, 1, -1), N(0, 0, -1), mat);
        quad(P(1, -1, 1), P(1, -1, -1), P(1, 1, -1), P(1, 1, 1), N(1, 0, 0), mat);
        quad(P(-1, -1, -1), P(-1, -1, 1), P(-1, 1, 1), P(-1, 1, -1), N(-1, 0, 0), mat);
        quad(P(-1, 1, 1), P(1, 1, 1), P(1, 1, -1), P(-1, 1, -1), N(0, 1, 0), mat);
        quad(P(-1, -1, -1), P(1, -1, -1), P(1, -1, 1), P(-1, -1, 1), N(0, -1, 0), mat);
    }
    // cylinder along +y, segments around, with caps
    void cylinder(V3 base, double r, double hgt, int seg, uint32_t mat) {
        for (int i = 0; i < seg; i++) {
            double a0 = 2 * M_PI * i / seg, a1 = 2 * M_PI * (i + 1) / seg;
            V3 n0{std::cos(a0), 0, std::sin(a0)}, n1{std::cos(a1), 0, std::sin(a1)};
            V3 b0 = base + n0 * r, b1 = base + n1 * r;
            V3 t0 = b0 + V3{0, hgt, 0}, t1 = b1 + V3{0, hgt, 0};
            tri(b0, b1, t1, n0, n1, n1, mat);
            tri(b0, t1, t0, n0, n1, n0, mat);
            V3 top = base + V3{0, hgt, 0};
            flat_tri(top, t1, t0, V3{0, 1, 0}, mat);
            flat_tri(base, b0, b1, V3{0, -1, 0}, mat);
        }
    }
    // UV sphere: stacks x slices, poles as fans
    void sphere(V3 c, double r, int stacks, int slices, uint32_t mat) {
        auto P = [&](int i, int j) {
            double th = M_PI * i / stacks, ph = 2 * M_PI * j / slices;
            return V3{std::sin(th) * std::cos(ph), std::cos(th), std::sin(th) * std::sin(ph)};
        };
        for (int i = 0; i < stacks; i++)
            for (int j = 0; j < slices; j++) {
                V3 a = P(i, j), b = P(i + 1, j), cc = P(i + 1, j + 1), d = P(i, j + 1);
                if (i != 0)
                    tri(c + a * r, c + b * r, c + d * r, a, b, d, mat);
                if (i != stacks - 1)
                    tri(c + d * r, c + b * r, c + cc * r, d, b, cc, mat);
            }
    }
    // half torus standing in the vertical plane through p0-p1 (an arch between two points)
    void arch(V3 p0, V3 p1, double minor, int seg_major, int seg_minor, uint32_t mat) {
        V3 mid = (p0 + p1) * 0.5;
        V3 ax = p1 - p0;
        double R = 0.5 * std::sqrt(vdot(ax, ax));
        V3 u = vnorm(ax), up{0, 1, 0};
        V3 w = vnorm(vcross(u, up));
        auto P = [&](int i, int j, V3 *n) {
            double a = M_PI * i / seg_major, b = 2 * M_PI * j / seg_minor;
            V3 radial = u * std::cos(a) + up * std::sin(a);
            V3 nn = radial * std::cos(b) + w * std::sin(b);
            *n = nn;
            return mid + radial * R + nn * minor;
        };
        for (int i = 0; i < seg_major; i++)
            for (int j = 0; j < seg_minor; j++) {
                V3 na, nb, nc, nd;
                V3 a = P(i, j, &na), b = P(i + 1, j, &nb), c = P(i + 1, j + 1, &nc), d = P(i, j + 1, &nd);
                tri(a, b, c, na, nb, nc, mat);
                tri(a, c, d, na, nc, nd, mat);
            }
    }
};

// Camera::Camera + focus + to_params (src/renderer/camera.cpp:3-56) with glm's float semantics:
// normalize(v) = v * (1/sqrt(dot)), radians(d) = d * 0.017453292...
void make_camera(const float pos[3], const float at[3], const float up[3], float hfov, float aspect, float defocus,
                 float focus, phx_camera_params *out) {
    struct G {
        float x, y, z;
    };
    auto sub = [](G a, G b) { return G{a.x - b.x, a.y - b.y, a.z - b.z}; };
    auto mul = [](G a, float s) { return G{a.x * s, a.y * s, a.z * s}; };
    auto dotg = [](G a, G b) { return a.x * b.x + a.y * b.y + a.z * b.z; };
    auto nrm = [&](G a) { return mul(a, 1.0f / std::sqrt(dotg(a, a))); };
    auto crs = [](G a, G b) { return G{a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y}; };
    const float deg2rad = (float)0.01745329251994329576923690768489;
    G P{pos[0], pos[1], pos[2]}, T{at[0], at[1], at[2]}, U{up[0], up[1], up[2]};
    float fd = 1.0f, da = 0.0f;
    G dd_u{0, 0, 0}, dd_v{0, 0, 0};
    G hor, ver, ll, uu, vv, ww;
    auto recalc = [&]() {
        ww = nrm(sub(P, T));
        uu = nrm(crs(U, ww));
        vv = crs(ww, uu);
        float hf = hfov * deg2rad;
        float hw = std::tan(hf * 0.5f) * fd;
        float hh = hw / aspect;
        hor = mul(uu, 2.0f * hw);
        ver = mul(vv, 2.0f * hh);
        ll = sub(sub(sub(P, mul(hor, 0.5f)), mul(ver, 0.5f)), mul(ww, fd));
    };
    recalc();
    // focus()
    da = defocus;
    fd = focus;
    float dr = fd * std::tan((da / 2.0f) * deg2rad);
    dd_u = mul(uu, dr);
    dd_v = mul(vv, dr);
    recalc();
    auto f4 = [](G g) { return phx_f4{g.x, g.y, g.z, 0.0f}; };
    std::memset(out, 0, sizeof(*out));
    out->position = f4(P);
    out->lower_left_corner = f4(ll);
    out->horizontal = f4(hor);
    out->vertical = f4(ver);
    out->defocus_disk_u = f4(dd_u);
    out->defocus_disk_v = f4(dd_v);
    out->defocus_angle = da;
    out->focus_distance = fd;
}

void finish_lights(SceneStore &s) { // SceneData::build_lum_pref_sum (scene_data.cpp:14-23)
    s.lum.clear();
    float run = 0.0f;
    for (const auto &l : s.lights) {
        float lum = l.power.x * 0.2126f + l.power.y * 0.7152f + l.power.z * 0.0722f;
        run += std::max(lum, 0.0f);
        s.lum.push_back(run);
    }
}

void cornell(Gen &g, bool with_light = true) {
    uint32_t white = g.material(make_material(0.73f, 0.71f, 0.68f, 0.0f, 1.0f));
    uint32_t red = g.material(make_material(0.63f, 0.06f, 0.04f, 0.0f, 1.0f));
    uint32_t green = g.material(make_material(0.14f, 0.45f, 0.09f, 0.0f, 1.0f));
    g.quad({0, 0, 0}, {1, 0, 0}, {1, 0, 1}, {0, 0, 1}, {0, 1, 0}, white);   // floor
    g.quad({0, 1, 0}, {0, 1, 1}, {1, 1, 1}, {1, 1, 0}, {0, -1, 0}, white);  // ceiling
    g.quad({0, 0, 0}, {0, 1, 0}, {1, 1, 0}, {1, 0, 0}, {0, 0, 1}, white);   // back
    g.quad({0, 0, 0}, {0, 0, 1}, {0, 1, 1}, {0, 1, 0}, {1, 0, 0}, red);     // left
    g.quad({1, 0, 0}, {1, 1, 0}, {1, 1, 1}, {1, 0, 1}, {-1, 0, 0}, green);  // right
    if (with_light) {
        phx_material lm = make_material(0.78f, 0.78f, 0.78f, 0.0f, 1.0f);
        lm.emissive = {15.0f, 15.0f, 15.0f, 0.0f};
        uint32_t light = g.material(lm);
        double y = 0.999, a = 0.375, b = 0.625;
        g.emissive_quad({a, y, a}, {a, y, b}, {b, y, b}, {b, y, a}, {0, -1, 0}, light, {15.0, 15.0, 15.0});
    }
}

void caustic_extras(Gen &g, Pcg &rng, uint32_t n_side, int sph_seg) {
    phx_material wm = make_material(1.0f, 1.0f, 1.0f, 0.0f, 0.05f);
    wm.transmission = 1.0f;
    wm.ior = 1.33f;
    uint32_t water = g.material(wm);
    uint32_t copper = g.material(make_material(0.95f, 0.64f, 0.54f, 1.0f, 0.2f));
    struct Wave {
        double a, k, dx, dz, ph;
    } w[8];
    for (auto &wv : w) {
        wv.a = rng.uni(0.002, 0.01);
        double lambda = rng.uni(0.05, 0.3);
        wv.k = 2 * M_PI / lambda;
        double th = rng.uni(0.0, 2 * M_PI);
        wv.dx = std::cos(th);
        wv.dz = std::sin(th);
        wv.ph = rng.uni(0.0, 2 * M_PI);
    }
    auto height = [&](double x, double z, double *gx, double *gz) {
        double h = 0.4;
        *gx = *gz = 0;
        for (auto &wv : w) {
            double arg = wv.k * (wv.dx * x + wv.dz * z) + wv.ph;
            h += wv.a * std::sin(arg);
            *gx += wv.a * wv.k * wv.dx * std::cos(arg);
            *gz += wv.a * wv.k * wv.dz * std::cos(arg);
        }
        return h;
    };
    std::vector<V3> P((size_t)n_side * n_side), N((size_t)n_side * n_side);
    for (uint32_t j = 0; j < n_side; j++)
        for (uint32_t i = 0; i < n_side; i++) {
            double x = (double)i / (n_side - 1), z = (double)j / (n_side - 1), gx, gz;
            double y = height(x, z, &gx, &gz);
            P[(size_t)j * n_side + i] = {x, y, z};
            N[(size_t)j * n_side + i] = vnorm(V3{-gx, 1.0, -gz});
        }
    for (uint32_t j = 0; j + 1 < n_side; j++)
        for (uint32_t i = 0; i + 1 < n_side; i++) {
            size_t a = (size_t)j * n_side + i, b = a + 1, c = a + n_side + 1, d = a + n_side;
            g.tri(P[a], P[d], P[c], N[a], N[d], N[c], water);
            g.tri(P[a], P[c], P[b], N[a], N[c], N[b], water);
        }
    g.sphere({0.66, 0.62, 0.42}, 0.15, sph_seg, sph_seg, copper);
}

void sky_envmap(SceneStore &s, uint32_t w, uint32_t h, V3 sun_dir) {
    // analytic sky: horizon-to-zenith gradient plus a Gaussian sun lobe; stored in the
    // reference's z-up equirect layout (envmap.h:9-20), scene up = +y
    s.env_w = w;
    s.env_h = h;
    s.envmap.resize((size_t)w * h * 3);
    V3 sd = vnorm(sun_dir);
    for (uint32_t py = 0; py < h; py++) {
        double v = (py + 0.5) / h;
        double theta = (1.0 - v) * M_PI; // v = 1 - theta/pi
        for (uint32_t px = 0; px < w; px++) {
            double u = (px + 0.5) / w;
            double phi = u * 2 * M_PI - M_PI;
            V3 d{std::sin(theta) * std::cos(phi), std::sin(theta) * std::sin(phi), std::cos(theta)};
            double up = d.y; // scene up
            double t = std::max(0.0, up);
            V3 horizon{0.9, 0.85, 0.8}, zenith{0.25, 0.45, 0.85}, ground{0.3, 0.28, 0.25};
            V3 c = up >= 0 ? horizon * (1 - t) + zenith * t : ground;
            double cosang = vdot(d, sd);
            double lobe = 40.0 * std::exp(-(1.0 - cosang) / 0.0015);
            float *o = &s.envmap[((size_t)py * w + px) * 3];
            o[0] = (float)(c.x + lobe * 1.0);
            o[1] = (float)(c.y + lobe * 0.95);
            o[2] = (float)(c.z + lobe * 0.85);
        }
    }
}

void atrium(Gen &g, Pcg &rng, int arch_seg, int env_w, int env_h) {
    std::vector<uint32_t> mats;
    for (int i = 0; i < 32; i++) {
        float r = (float)rng.uni(0.05, 0.9), gg = (float)rng.uni(0.05, 0.9), b = (float)rng.uni(0.05, 0.9);
        float rough = (float)rng.uni(0.05, 0.9);
        float metal = rng.uni() < 0.3 ? 1.0f : 0.0f;
        mats.push_back(g.material(make_material(r, gg, b, metal, rough)));
    }
    auto pick = [&]() { return mats[rng.next() % 32u]; };
    double X = 8, Z = 6;
    g.quad({-12, 0, -10}, {-12, 0, 10}, {12, 0, 10}, {12, 0, -10}, {0, 1, 0}, mats[0]);
    // 24 columns around the courtyard perimeter: 8 per long side, 4 per short side (corners shared)
    std::vector<V3> ring;
    for (int i = 0; i < 8; i++)
        ring.push_back({-X + 2 * X * i / 7.0, 0, -Z});
    for (int i = 1; i <= 4; i++)
        ring.push_back({X, 0, -Z + 2 * Z * i / 5.0});
    for (int i = 7; i >= 0; i--)
        ring.push_back({-X + 2 * X * i / 7.0, 0, Z});
    for (int i = 4; i >= 1; i--)
        ring.push_back({-X, 0, -Z + 2 * Z * i / 5.0});
    const double col_r = 0.35, col_h = 4.0, slab_y = 5.3, slab_t = 0.3;
    const double floors[2] = {0.0, slab_y + slab_t};
    int minor_seg = std::max(8, arch_seg * 40 / 64);
    for (double fy : floors) {
        uint32_t cm = pick(), am = pick();
        for (const V3 &p : ring)
            g.cylinder({p.x, fy, p.z}, col_r, col_h, 64, cm);
        for (size_t i = 0; i < ring.size(); i++) {
            const V3 &a = ring[i], &b = ring[(i + 1) % ring.size()];
            g.arch({a.x, fy + col_h, a.z}, {b.x, fy + col_h, b.z}, 0.25, arch_seg, minor_seg, am);
        }
    }
    uint32_t sm = pick();
    g.box({-X - 0.6, slab_y, -Z - 0.6}, {X + 0.6, slab_y + slab_t, -Z + 0.6}, 0, sm);
    g.box({-X - 0.6, slab_y, Z - 0.6}, {X + 0.6, slab_y + slab_t, Z + 0.6}, 0, sm);
    g.box({-X - 0.6, slab_y, -Z + 0.6}, {-X + 0.6, slab_y + slab_t, Z - 0.6}, 0, sm);
    g.box({X - 0.6, slab_y, -Z + 0.6}, {X + 0.6, slab_y + slab_t, Z - 0.6}, 0, sm);
    for (int i = 0; i < 400; i++) {
        double sx = rng.uni(0.05, 0.5), sy = rng.uni(0.05, 0.5), sz = rng.uni(0.05, 0.5);
        double cx = rng.uni(-X + 1, X - 1), cz = rng.uni(-Z + 1, Z - 1), yaw = rng.uni(0, M_PI);
        g.box({cx - sx / 2, 0, cz - sz / 2}, {cx + sx / 2, sy, cz + sz / 2}, yaw, pick());
    }
    phx_light sun{};
    sun.kind = PHX_LIGHT_POINT;
    V3 sun_pos{2.0, 14.0, 3.0};
    sun.position = F4(sun_pos);
    sun.power = {200.0f, 190.0f, 170.0f, 0.0f};
    g.s.lights.push_back(sun);
    sky_envmap(g.s, (uint32_t)env_w, (uint32_t)env_h, sun_pos);
}

} // namespace

int scene_generate(const phx_scene_spec &spec, SceneStore &s, std::string &err) {
    s = SceneStore{};
    Gen g(s);
    Pcg rng(spec.seed);
    float aspect = spec.height ? (float)spec.width / (float)spec.height : 1.0f;
    switch (spec.kind) {
    case PHX_SCENE_CORNELL: {
        cornell(g);
        float pos[3] = {0.5f, 0.5f, 2.4f}, at[3] = {0.5f, 0.5f, 0.0f}, up[3] = {0.0f, 1.0f, 0.0f};
        make_camera(pos, at, up, 40.0f, aspect, 0.0f, 1.0f, &s.camera);
        break;
    }
    case PHX_SCENE_CAUSTIC: {
        cornell(g);
        uint32_t side = spec.detail ? spec.detail : 256u;
        if (side < 2)
            side = 2;
        int seg = spec.detail ? std::max(6, (int)(side * 100 / 256)) : 100;
        caustic_extras(g, rng, side, seg);
        float pos[3] = {0.5f, 0.5f, 2.4f}, at[3] = {0.5f, 0.5f, 0.0f}, up[3] = {0.0f, 1.0f, 0.0f};
        make_camera(pos, at, up, 40.0f, aspect, 0.0f, 1.0f, &s.camera);
        break;
    }
    case PHX_SCENE_ATRIUM: {
        int seg = spec.detail ? (int)spec.detail : 64;
        int ew = spec.detail ? 512 : 2048, eh = spec.detail ? 256 : 1024;
        atrium(g, rng, std::max(4, seg), ew, eh);
        float pos[3] = {-6.2f, 1.7f, -4.6f}, at[3] = {5.0f, 3.2f, 4.0f}, up[3] = {0.0f, 1.0f, 0.0f};
        make_camera(pos, at, up, 75.0f, aspect, 0.0f, 1.0f, &s.camera);
        break;
    }
    default:
        err = "unknown scene kind";
        return PHX_E_INVALID;
    }
    finish_lights(s);
    return PHX_OK;
}

} // namespace phx

namespace phx {
int camera_make(const float p[3], const float a[3], const float u[3], float hfov, float aspect, float defocus,
                float focus, phx_camera_params *out) {
    make_camera(p, a, u, hfov, aspect, defocus, focus, out);
    return PHX_OK;
}
void lum_pref_sum(const phx_light *l, uint32_t n, float *out) {
    float run = 0.0f;
    for (uint32_t i = 0; i < n; i++) {
        float lum = l[i].power.x * 0.2126f + l[i].power.y * 0.7152f + l[i].power.z * 0.0722f;
        run += std::max(lum, 0.0f);
        out[i] = run;
    }
}
} // namespace phx
