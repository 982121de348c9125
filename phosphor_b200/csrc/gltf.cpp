// gltf.cpp — glTF 2.0 scene ingest: the reference's read_gltf_scene (src/parsers/scene.cpp:206-233,
// parse_node/_mesh/_camera/_light :36-204, material.cpp:9-184, texture.cpp:19-92), which reads
// .gltf/.glb files through assimp, restated directly over the glTF 2.0 document (assimp is not
// used).  What the reference takes from assimp is taken from the glTF document with glTF's
// definitions and defaults:
//   * nodes: matrix or translation·rotation·scale, composed parent·local from the default scene's
//     roots; per node its camera, its KHR_lights_punctual light, then its mesh's primitives (one
//     mesh each, as assimp splits them), then its children — the reference's traversal order;
//   * primitives: triangles, triangle strips and fans (the strip's odd triangles reversed, as
//     glTF specifies), indexed or not; POSITION, NORMAL, TANGENT (xyz) and TEXCOORD_0 of any
//     accessor component type (normalized integers scaled to [0, 1]); points and lines are
//     skipped; texture coordinates are flipped to (u, 1 - v), the image-row convention the
//     reference's sampler expects (material.h:105-107 flips v back);
//   * positions by the node transform, normals and tangents by its inverse transpose, normalized;
//     a missing normal becomes the face normal and a missing tangent the reference's face tangent
//     from the UVs (scene.cpp:64-95) — assimp would derive per-vertex tangents here instead;
//   * materials: one per primitive (scene.cpp:40, material.cpp:157-184), from
//     pbrMetallicRoughness (baseColorFactor, metallicFactor, roughnessFactor: glTF defaults 1),
//     emissiveFactor × KHR_materials_emissive_strength, KHR_materials_transmission,
//     KHR_materials_ior, KHR_materials_volume (thickness, attenuation distance and colour), the
//     base-colour, emissive, normal, occlusion, metallic-roughness and transmission textures and
//     their KHR_texture_transform offset, scale and rotation (rotation negated, offset moved, for
//     the flipped v); a primitive without material gets the reference's default material;
//   * an emissive material (a component above 1e-5) makes its triangles emissive triangles and one
//     textured area light of power π·emissive·area (scene.cpp:117-130);
//   * cameras: perspective; position, -z view and +y up by the node transform; horizontal field
//     of view 2·atan(aspectRatio·tan(yfov/2)); the render's width/height then replace the aspect
//     and focus() applies the defocus angle and focus distance (renderer.cpp:24-28);
//   * lights: power = colour × intensity / 683 (scene.cpp:143-148); point, spot (inner and
//     outer cone angles) and directional, pointing along -z by the node's rotation;
//   * textures: images in the reference's load order (per material: base colour, emissive,
//     normal, occlusion, metallic-roughness, transmission; texture.cpp:80-92), each once, as
//     8-bit RGB; PNG from files, data URIs or buffer views is decoded, other formats are
//     skipped (the material then has no texture, as when the reference fails to load one).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>

#include "host.hpp"
#include "json_min.hpp"
#include "png_min.hpp"

namespace phx {
namespace {

constexpr float EPS_F = 1e-5f;
constexpr float PI_F = 3.141592654f;
constexpr float LUMINOUS_EFFICACY = 683.0f;

struct F3 {
    float x, y, z;
};
inline F3 sub(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline F3 add(F3 a, F3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline F3 mul(F3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline F3 crossf(F3 a, F3 b) { return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y}; }
inline float dotf(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline F3 normf(F3 a) { return mul(a, 1.0f / std::sqrt(dotf(a, a))); }
inline phx_f4 f4(F3 v) { return {v.x, v.y, v.z, 0.0f}; }

// 4x4 column-major (m[col * 4 + row]), like the glTF node matrix
struct M4 {
    float m[16];
};
M4 ident() {
    M4 r{};
    r.m[0] = r.m[5] = r.m[10] = r.m[15] = 1.0f;
    return r;
}
M4 mulm(const M4 &a, const M4 &b) {
    M4 r{};
    for (int c = 0; c < 4; c++)
        for (int rr = 0; rr < 4; rr++) {
            float s = 0.0f;
            for (int k = 0; k < 4; k++)
                s += a.m[k * 4 + rr] * b.m[c * 4 + k];
            r.m[c * 4 + rr] = s;
        }
    return r;
}
F3 xpoint(const M4 &a, F3 p) {
    return {a.m[0] * p.x + a.m[4] * p.y + a.m[8] * p.z + a.m[12], a.m[1] * p.x + a.m[5] * p.y + a.m[9] * p.z + a.m[13],
            a.m[2] * p.x + a.m[6] * p.y + a.m[10] * p.z + a.m[14]};
}
F3 xdir(const M4 &a, F3 d) {
    return {a.m[0] * d.x + a.m[4] * d.y + a.m[8] * d.z, a.m[1] * d.x + a.m[5] * d.y + a.m[9] * d.z,
            a.m[2] * d.x + a.m[6] * d.y + a.m[10] * d.z};
}
// inverse transpose of the upper 3x3, as a row-major 3x3 applied to column vectors
struct M3 {
    float r[9];
};
M3 normal_matrix(const M4 &a) {
    const float m00 = a.m[0], m10 = a.m[1], m20 = a.m[2], m01 = a.m[4], m11 = a.m[5], m21 = a.m[6], m02 = a.m[8],
                m12 = a.m[9], m22 = a.m[10];
    const float c00 = m11 * m22 - m12 * m21, c01 = m12 * m20 - m10 * m22, c02 = m10 * m21 - m11 * m20;
    const float c10 = m02 * m21 - m01 * m22, c11 = m00 * m22 - m02 * m20, c12 = m01 * m20 - m00 * m21;
    const float c20 = m01 * m12 - m02 * m11, c21 = m02 * m10 - m00 * m12, c22 = m00 * m11 - m01 * m10;
    const float det = m00 * c00 + m01 * c01 + m02 * c02;
    const float inv = det != 0.0f ? 1.0f / det : 0.0f;
    // (A^-1)^T = cofactor(A) / det
    return M3{{c00 * inv, c01 * inv, c02 * inv, c10 * inv, c11 * inv, c12 * inv, c20 * inv, c21 * inv, c22 * inv}};
}
F3 xnormal(const M3 &n, F3 v) {
    return {n.r[0] * v.x + n.r[1] * v.y + n.r[2] * v.z, n.r[3] * v.x + n.r[4] * v.y + n.r[5] * v.z,
            n.r[6] * v.x + n.r[7] * v.y + n.r[8] * v.z};
}

M4 node_matrix(const Json &n) {
    M4 r = ident();
    if (n.has("matrix") && n["matrix"].size() == 16) {
        for (int i = 0; i < 16; i++)
            r.m[i] = (float)n["matrix"][i].number(0.0);
        return r;
    }
    float t[3] = {0, 0, 0}, q[4] = {0, 0, 0, 1}, s[3] = {1, 1, 1};
    for (int i = 0; i < 3; i++) {
        t[i] = (float)n["translation"][i].number(0.0);
        s[i] = (float)n["scale"][i].number(1.0);
    }
    for (int i = 0; i < 4; i++)
        q[i] = (float)n["rotation"][i].number(i == 3 ? 1.0 : 0.0);
    const float x = q[0], y = q[1], z = q[2], w = q[3];
    const float R[9] = {1 - 2 * (y * y + z * z), 2 * (x * y + z * w), 2 * (x * z - y * w),   // column 0
                        2 * (x * y - z * w), 1 - 2 * (x * x + z * z), 2 * (y * z + x * w),   // column 1
                        2 * (x * z + y * w), 2 * (y * z - x * w), 1 - 2 * (x * x + y * y)};  // column 2
    for (int c = 0; c < 3; c++)
        for (int rr = 0; rr < 3; rr++)
            r.m[c * 4 + rr] = R[c * 3 + rr] * s[c];
    r.m[12] = t[0];
    r.m[13] = t[1];
    r.m[14] = t[2];
    return r;
}

bool read_file(const std::string &path, std::vector<uint8_t> &out) {
    std::ifstream f(path, std::ios::binary);
    if (!f)
        return false;
    out.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
    return true;
}

bool base64(const std::string &s, size_t from, std::vector<uint8_t> &out) {
    auto val = [](char c) -> int {
        if (c >= 'A' && c <= 'Z')
            return c - 'A';
        if (c >= 'a' && c <= 'z')
            return c - 'a' + 26;
        if (c >= '0' && c <= '9')
            return c - '0' + 52;
        if (c == '+' || c == '-')
            return 62;
        if (c == '/' || c == '_')
            return 63;
        return -1;
    };
    uint32_t acc = 0;
    int bits = 0;
    out.clear();
    for (size_t i = from; i < s.size(); i++) {
        if (s[i] == '=')
            break;
        int v = val(s[i]);
        if (v < 0)
            return false;
        acc = (acc << 6) | (uint32_t)v;
        bits += 6;
        if (bits >= 8) {
            bits -= 8;
            out.push_back((uint8_t)(acc >> bits));
        }
    }
    return true;
}

std::string uri_decode(const std::string &u) {
    std::string r;
    for (size_t i = 0; i < u.size(); i++) {
        if (u[i] == '%' && i + 2 < u.size()) {
            r += (char)std::stoi(u.substr(i + 1, 2), nullptr, 16);
            i += 2;
        } else {
            r += u[i];
        }
    }
    return r;
}

struct Doc {
    Json j;
    std::vector<std::vector<uint8_t>> buffers;
    std::string dir;

    // raw bytes of a URI: data URI (base64) or a file beside the document
    bool uri_bytes(const std::string &uri, std::vector<uint8_t> &out) const {
        if (uri.rfind("data:", 0) == 0) {
            size_t comma = uri.find(',');
            return comma != std::string::npos && uri.find(";base64") < comma && base64(uri, comma + 1, out);
        }
        return read_file(dir + "/" + uri_decode(uri), out);
    }
    bool view_bytes(int64_t view, const uint8_t **p, size_t *n, size_t *stride) const {
        const Json &bv = j["bufferViews"][(size_t)view];
        const int64_t b = bv["buffer"].integer(-1);
        if (b < 0 || (size_t)b >= buffers.size())
            return false;
        const size_t off = (size_t)bv["byteOffset"].integer(0), len = (size_t)bv["byteLength"].integer(0);
        if (off + len > buffers[(size_t)b].size())
            return false;
        *p = buffers[(size_t)b].data() + off;
        *n = len;
        *stride = (size_t)bv["byteStride"].integer(0);
        return true;
    }
    // accessor as floats (ncomp per element); integer components are scaled to [0, 1] when normalized
    bool accessor(int64_t idx, std::vector<float> &out, int *ncomp, std::string &err) const {
        const Json &a = j["accessors"][(size_t)idx];
        if (a.kind != Json::Object) {
            err = "accessor " + std::to_string(idx) + " missing";
            return false;
        }
        if (a.has("sparse")) {
            err = "sparse accessors are not supported";
            return false;
        }
        static const std::map<std::string, int> comps = {{"SCALAR", 1}, {"VEC2", 2}, {"VEC3", 3}, {"VEC4", 4}};
        auto it = comps.find(a["type"].string());
        if (it == comps.end()) {
            err = "unsupported accessor type " + a["type"].string();
            return false;
        }
        const int nc = it->second;
        const int64_t ct = a["componentType"].integer(0);
        const size_t csize = (ct == 5120 || ct == 5121) ? 1 : (ct == 5122 || ct == 5123) ? 2 : (ct == 5125 || ct == 5126) ? 4 : 0;
        if (!csize) {
            err = "unsupported component type";
            return false;
        }
        const size_t count = (size_t)a["count"].integer(0);
        const bool norm = a["normalized"].kind == Json::Bool && a["normalized"].b;
        out.assign(count * nc, 0.0f);
        *ncomp = nc;
        if (!a.has("bufferView"))
            return true; // all zero (glTF: no buffer view means zeros)
        const uint8_t *p;
        size_t n, stride;
        if (!view_bytes(a["bufferView"].integer(-1), &p, &n, &stride)) {
            err = "bad buffer view";
            return false;
        }
        const size_t off = (size_t)a["byteOffset"].integer(0), elem = csize * nc;
        if (!stride)
            stride = elem;
        if (count && off + (count - 1) * stride + elem > n) {
            err = "accessor runs past its buffer view";
            return false;
        }
        for (size_t e = 0; e < count; e++)
            for (int c = 0; c < nc; c++) {
                const uint8_t *q = p + off + e * stride + c * csize;
                float v;
                switch (ct) {
                case 5126: std::memcpy(&v, q, 4); break;
                case 5125: { uint32_t u; std::memcpy(&u, q, 4); v = (float)u; break; }
                case 5123: { uint16_t u; std::memcpy(&u, q, 2); v = norm ? u / 65535.0f : (float)u; break; }
                case 5122: { int16_t u; std::memcpy(&u, q, 2); v = norm ? std::max(u / 32767.0f, -1.0f) : (float)u; break; }
                case 5121: v = norm ? q[0] / 255.0f : (float)q[0]; break;
                default: { int8_t u = (int8_t)q[0]; v = norm ? std::max(u / 127.0f, -1.0f) : (float)u; break; }
                }
                out[e * nc + c] = v;
            }
        return true;
    }
    bool indices(int64_t idx, std::vector<uint32_t> &out, std::string &err) const {
        const Json &a = j["accessors"][(size_t)idx];
        const int64_t ct = a["componentType"].integer(0);
        if (ct != 5121 && ct != 5123 && ct != 5125) {
            err = "index accessor must be an unsigned integer type";
            return false;
        }
        std::vector<float> f;
        int nc;
        if (!accessor(idx, f, &nc, err))
            return false;
        out.resize(f.size());
        if (ct == 5125 && a.has("bufferView")) { // re-read exactly (a float holds 24 bits)
            const uint8_t *p;
            size_t n, stride;
            if (!view_bytes(a["bufferView"].integer(-1), &p, &n, &stride)) {
                err = "bad buffer view";
                return false;
            }
            const size_t off = (size_t)a["byteOffset"].integer(0);
            for (size_t i = 0; i < out.size(); i++)
                std::memcpy(&out[i], p + off + i * (stride ? stride : 4), 4);
        } else {
            for (size_t i = 0; i < out.size(); i++)
                out[i] = (uint32_t)f[i];
        }
        return true;
    }
};

phx_material default_material() { // material.cpp:9-30
    phx_material m{};
    m.base_color = {1.0f, 1.0f, 1.0f, 1.0f};
    m.emissive = {0.0f, 0.0f, 0.0f, 0.0f};
    m.metallic = 0.0f;
    m.roughness = 1.0f;
    m.transmission = 0.0f;
    m.ior = 1.5f;
    m.diff_index = m.emis_index = m.norm_index = m.occlusion_index = m.metal_rough_index = m.transmission_index =
        PHX_NO_TEXTURE;
    m.att_color = {1.0f, 1.0f, 1.0f, 0.0f};
    m.att_dist = 1e9f;
    m.thickness = 0.0f;
    return m;
}

phx_uv_transform_block default_uv() { // material.cpp:32-48
    phx_uv_transform id{};
    id.uv_offset = {0.0f, 0.0f};
    id.uv_scale = {1.0f, 1.0f};
    id.uv_rotation = 0.0f;
    phx_uv_transform_block b{};
    b.diff = b.emis = b.norm = b.occlusion = b.metal_rough = b.transmission = id;
    return b;
}

struct Loader {
    const Doc &d;
    SceneStore &s;
    std::map<int64_t, uint32_t> tex_of_image; // glTF image index -> atlas texture
    std::vector<phx_f4> cams_pos, cams_at, cams_up;
    std::vector<float> cams_hfov, cams_aspect;
    std::string err;
    uint32_t skipped_textures = 0;

    Loader(const Doc &doc, SceneStore &st) : d(doc), s(st) {}

    int64_t image_of(const Json &texinfo) const {
        if (texinfo.kind != Json::Object)
            return -1;
        const Json &t = d.j["textures"][(size_t)texinfo["index"].integer(-1)];
        return t["source"].integer(-1);
    }
    // texture.cpp:19-78: decode once, 8-bit RGB, appended to the atlas
    void load_image(int64_t img) {
        if (img < 0 || tex_of_image.count(img))
            return;
        const Json &im = d.j["images"][(size_t)img];
        std::vector<uint8_t> bytes;
        bool ok = false;
        if (im.has("uri")) {
            ok = d.uri_bytes(im["uri"].string(), bytes);
        } else if (im.has("bufferView")) {
            const uint8_t *p;
            size_t n, stride;
            if (d.view_bytes(im["bufferView"].integer(-1), &p, &n, &stride)) {
                bytes.assign(p, p + n);
                ok = true;
            }
        }
        std::vector<uint8_t> rgb;
        uint32_t w = 0, h = 0;
        std::string why;
        if (!ok || !png_decode_rgb8(bytes.data(), bytes.size(), rgb, &w, &h, why)) {
            skipped_textures++;
            return;
        }
        phx_texture_meta m{};
        m.atlas_offset = (uint32_t)s.atlas.size();
        m.width = w;
        m.height = h;
        m.channels = 3;
        s.atlas.insert(s.atlas.end(), rgb.begin(), rgb.end());
        tex_of_image[img] = (uint32_t)s.tex_meta.size();
        s.tex_meta.push_back(m);
    }
    static std::vector<const Json *> texinfos(const Json &m) {
        const Json &pbr = m["pbrMetallicRoughness"];
        const Json &ext = m["extensions"];
        return {&pbr["baseColorTexture"], &m["emissiveTexture"], &m["normalTexture"], &m["occlusionTexture"],
                &pbr["metallicRoughnessTexture"], &ext["KHR_materials_transmission"]["transmissionTexture"]};
    }
    void load_textures() { // texture.cpp:80-92
        for (size_t i = 0; i < d.j["materials"].size(); i++)
            for (const Json *ti : texinfos(d.j["materials"][i]))
                load_image(image_of(*ti));
    }
    uint32_t tex_index(const Json &texinfo) const {
        auto it = tex_of_image.find(image_of(texinfo));
        return it == tex_of_image.end() ? PHX_NO_TEXTURE : it->second;
    }
    // KHR_texture_transform for the flipped v: the transform T·R(r)·S of the glTF coordinate, seen
    // from (u, 1 - v), is R(-r)·S of it plus a moved offset
    static void uv_transform(const Json &texinfo, phx_uv_transform &t) {
        const Json &x = texinfo["extensions"]["KHR_texture_transform"];
        if (x.kind != Json::Object)
            return;
        const float ox = (float)x["offset"][0].number(0.0), oy = (float)x["offset"][1].number(0.0);
        const float sx = (float)x["scale"][0].number(1.0), sy = (float)x["scale"][1].number(1.0);
        const float r = (float)x["rotation"].number(0.0);
        const float c = std::cos(r), sn = std::sin(r);
        // glTF: u' = c·sx·u + sn·sy·v + ox, v' = -sn·sx·u + c·sy·v + oy.  With U = u, V = 1 - v and the
        // result's v flipped back: U' = c·sx·U - sn·sy·V + (sn·sy + ox), V' = sn·sx·U + c·sy·V + (1 - c·sy - oy)
        t.uv_scale = {sx, sy};
        t.uv_rotation = r;
        t.uv_offset = {sn * sy + ox, 1.0f - c * sy - oy};
    }

    // material.cpp:157-184 (one material per primitive)
    uint32_t material(int64_t mi, F3 *emissive) {
        phx_material m = default_material();
        phx_uv_transform_block uv = default_uv();
        *emissive = {0, 0, 0};
        const Json &jm = d.j["materials"][(size_t)std::max<int64_t>(mi, 0)];
        if (mi >= 0 && jm.kind == Json::Object) {
            const Json &pbr = jm["pbrMetallicRoughness"];
            for (int c = 0; c < 4; c++)
                (&m.base_color.x)[c] = (float)pbr["baseColorFactor"][c].number(1.0);
            m.metallic = (float)pbr["metallicFactor"].number(1.0);
            m.roughness = (float)pbr["roughnessFactor"].number(1.0);
            const float strength = (float)jm["extensions"]["KHR_materials_emissive_strength"]["emissiveStrength"].number(1.0);
            F3 e{(float)jm["emissiveFactor"][0].number(0.0), (float)jm["emissiveFactor"][1].number(0.0),
                 (float)jm["emissiveFactor"][2].number(0.0)};
            e = mul(e, strength);
            m.emissive = f4(e);
            const Json &ext = jm["extensions"];
            m.transmission = (float)ext["KHR_materials_transmission"]["transmissionFactor"].number(0.0);
            m.ior = (float)ext["KHR_materials_ior"]["ior"].number(1.5);
            const Json &vol = ext["KHR_materials_volume"];
            m.thickness = (float)vol["thicknessFactor"].number(0.0);
            m.att_dist = (float)vol["attenuationDistance"].number(1e9);
            if (vol["attenuationColor"].kind == Json::Array)
                m.att_color = {(float)vol["attenuationColor"][0].number(1.0), (float)vol["attenuationColor"][1].number(1.0),
                               (float)vol["attenuationColor"][2].number(1.0), 1.0f};
            const auto ti = texinfos(jm);
            m.diff_index = tex_index(*ti[0]);
            m.emis_index = tex_index(*ti[1]);
            m.norm_index = tex_index(*ti[2]);
            m.occlusion_index = tex_index(*ti[3]);
            m.metal_rough_index = tex_index(*ti[4]);
            m.transmission_index = tex_index(*ti[5]);
            uv_transform(*ti[0], uv.diff);
            uv_transform(*ti[1], uv.emis);
            uv_transform(*ti[2], uv.norm);
            uv_transform(*ti[3], uv.occlusion);
            uv_transform(*ti[4], uv.metal_rough);
            uv_transform(*ti[5], uv.transmission);
            if (e.x > EPS_F || e.y > EPS_F || e.z > EPS_F)
                *emissive = e;
        }
        s.mats.push_back(m);
        s.uvs.push_back(uv);
        return (uint32_t)s.mats.size() - 1;
    }

    // scene.cpp:36-131
    bool primitive(const Json &p, const M4 &g) {
        const int64_t mode = p["mode"].integer(4);
        if (mode != 4 && mode != 5 && mode != 6)
            return true; // points and lines: no triangles
        const Json &at = p["attributes"];
        if (!at.has("POSITION")) {
            err = "primitive without POSITION";
            return false;
        }
        std::vector<float> pos, nrm, tan, uv;
        int nc = 0;
        if (!d.accessor(at["POSITION"].integer(-1), pos, &nc, err) || nc != 3)
            return err.empty() ? (err = "POSITION must be VEC3", false) : false;
        const size_t nv = pos.size() / 3;
        bool has_n = at.has("NORMAL"), has_t = at.has("TANGENT"), has_uv = at.has("TEXCOORD_0");
        if (has_n && (!d.accessor(at["NORMAL"].integer(-1), nrm, &nc, err) || nc != 3 || nrm.size() != 3 * nv))
            return err.empty() ? (err = "bad NORMAL", false) : false;
        int tc = 0;
        if (has_t && (!d.accessor(at["TANGENT"].integer(-1), tan, &tc, err) || tc < 3 || tan.size() != tc * nv))
            return err.empty() ? (err = "bad TANGENT", false) : false;
        if (has_uv && (!d.accessor(at["TEXCOORD_0"].integer(-1), uv, &nc, err) || nc != 2 || uv.size() != 2 * nv))
            return err.empty() ? (err = "bad TEXCOORD_0", false) : false;
        std::vector<uint32_t> idx;
        if (p.has("indices")) {
            if (!d.indices(p["indices"].integer(-1), idx, err))
                return false;
        } else {
            idx.resize(nv);
            for (size_t i = 0; i < nv; i++)
                idx[i] = (uint32_t)i;
        }
        for (uint32_t i : idx)
            if (i >= nv) {
                err = "index out of range";
                return false;
            }
        std::vector<uint32_t> tri;
        if (mode == 4) {
            tri.assign(idx.begin(), idx.begin() + (idx.size() / 3) * 3);
        } else if (mode == 5) {
            for (size_t i = 0; i + 2 < idx.size(); i++) {
                const bool odd = i % 2;
                tri.insert(tri.end(), {idx[i + (odd ? 1 : 0)], idx[i + (odd ? 0 : 1)], idx[i + 2]});
            }
        } else {
            for (size_t i = 1; i + 1 < idx.size(); i++)
                tri.insert(tri.end(), {idx[i], idx[i + 1], idx[0]});
        }
        F3 emissive;
        const uint32_t mat = material(p["material"].integer(-1), &emissive);
        const M3 nm = normal_matrix(g);
        const uint32_t start = (uint32_t)s.tris.size();
        auto P3 = [&](const std::vector<float> &a, uint32_t i, int k) { return F3{a[k * i], a[k * i + 1], a[k * i + 2]}; };
        for (size_t f = 0; f + 2 < tri.size(); f += 3) {
            const uint32_t i0 = tri[f], i1 = tri[f + 1], i2 = tri[f + 2];
            const F3 p0 = xpoint(g, P3(pos, i0, 3)), p1 = xpoint(g, P3(pos, i1, 3)), p2 = xpoint(g, P3(pos, i2, 3));
            float u[3][2] = {{0, 0}, {0, 0}, {0, 0}};
            if (has_uv) {
                const uint32_t ii[3] = {i0, i1, i2};
                for (int k = 0; k < 3; k++) {
                    u[k][0] = uv[2 * ii[k]];
                    u[k][1] = 1.0f - uv[2 * ii[k] + 1];
                }
            }
            F3 n0, n1, n2;
            if (has_n) {
                n0 = normf(xnormal(nm, P3(nrm, i0, 3)));
                n1 = normf(xnormal(nm, P3(nrm, i1, 3)));
                n2 = normf(xnormal(nm, P3(nrm, i2, 3)));
            } else {
                n0 = n1 = n2 = normf(crossf(sub(p1, p0), sub(p2, p0)));
            }
            F3 t0, t1, t2;
            if (has_t) {
                t0 = normf(xnormal(nm, P3(tan, i0, tc)));
                t1 = normf(xnormal(nm, P3(tan, i1, tc)));
                t2 = normf(xnormal(nm, P3(tan, i2, tc)));
            } else { // scene.cpp:83-95
                const F3 e1 = sub(p1, p0), e2 = sub(p2, p0);
                const float du1 = u[1][0] - u[0][0], dv1 = u[1][1] - u[0][1], du2 = u[2][0] - u[0][0],
                            dv2 = u[2][1] - u[0][1];
                const float det = du1 * dv2 - du2 * dv1;
                F3 ft{1.0f, 0.0f, 0.0f};
                if (!(std::fabs(det) < EPS_F)) {
                    const float inv = 1.0f / det;
                    ft = mul(sub(mul(e1, dv2), mul(e2, dv1)), inv);
                }
                t0 = t1 = t2 = normf(xnormal(nm, ft));
            }
            phx_triangle t{};
            t.v0 = f4(p0);
            t.v1 = f4(p1);
            t.v2 = f4(p2);
            t.n0 = f4(n0);
            t.n1 = f4(n1);
            t.n2 = f4(n2);
            t.t0 = f4(t0);
            t.t1 = f4(t1);
            t.t2 = f4(t2);
            t.uv0 = {u[0][0], u[0][1]};
            t.uv1 = {u[1][0], u[1][1]};
            t.uv2 = {u[2][0], u[2][1]};
            t.mat_index = mat;
            s.tris.push_back(t);
        }
        const uint32_t count = (uint32_t)s.tris.size() - start;
        if ((emissive.x > EPS_F || emissive.y > EPS_F || emissive.z > EPS_F) && count > 0) {
            const uint32_t estart = (uint32_t)s.etris.size();
            float area = 0.0f;
            for (uint32_t j = start; j < start + count; j++) {
                const phx_triangle &t = s.tris[j];
                s.etris.push_back(t);
                const F3 e1{t.v1.x - t.v0.x, t.v1.y - t.v0.y, t.v1.z - t.v0.z};
                const F3 e2{t.v2.x - t.v0.x, t.v2.y - t.v0.y, t.v2.z - t.v0.z};
                const F3 c = crossf(e1, e2);
                area += 0.5f * std::sqrt(dotf(c, c));
            }
            phx_light l{};
            l.kind = PHX_LIGHT_TEXTURED;
            l.power = f4(mul(mul(emissive, PI_F), area)); // PI * emissive * total_area
            uint32_t aux[3] = {s.mats[mat].emis_index, estart, count};
            std::memcpy(&l.aux, aux, 12);
            l.aux.w = area;
            s.lights.push_back(l);
        }
        return true;
    }

    void camera(const Json &c, const M4 &g) { // scene.cpp:133-150
        if (c["type"].string() != "perspective")
            return;
        const Json &pp = c["perspective"];
        const float yfov = (float)pp["yfov"].number(0.0), aspect = (float)pp["aspectRatio"].number(0.0);
        const F3 pos = xpoint(g, {0, 0, 0});
        const F3 look = xdir(g, {0, 0, -1});
        const F3 up = normf(xdir(g, {0, 1, 0}));
        cams_pos.push_back(f4(pos));
        cams_at.push_back(f4(add(pos, look)));
        cams_up.push_back(f4(up));
        cams_hfov.push_back(2.0f * std::atan(aspect * std::tan(yfov * 0.5f)) * (180.0f / PI_F));
        cams_aspect.push_back(aspect);
    }

    void light(const Json &l, const M4 &g) { // scene.cpp:152-181, light.cpp:4-45
        const F3 col{(float)l["color"][0].number(1.0), (float)l["color"][1].number(1.0), (float)l["color"][2].number(1.0)};
        const float intensity = (float)l["intensity"].number(1.0);
        const F3 ci = mul(col, intensity);
        const F3 power{ci.x / LUMINOUS_EFFICACY, ci.y / LUMINOUS_EFFICACY, ci.z / LUMINOUS_EFFICACY};
        const F3 pos = xpoint(g, {0, 0, 0});
        const std::string type = l["type"].string();
        phx_light out{};
        out.power = f4(power);
        if (type == "point") {
            out.kind = PHX_LIGHT_POINT;
            out.position = f4(pos);
        } else if (type == "spot") {
            const F3 dir = normf(xdir(g, {0, 0, -1}));
            out.kind = PHX_LIGHT_SPOT;
            out.position = f4(pos);
            out.direction = f4(dir);
            out.aux = {(float)l["spot"]["innerConeAngle"].number(0.0),
                       (float)l["spot"]["outerConeAngle"].number(PI_F / 4.0), 0.0f, 0.0f};
        } else if (type == "directional") {
            const F3 dir = normf(xdir(g, {0, 0, -1}));
            out.kind = PHX_LIGHT_DIRECTIONAL;
            out.direction = f4(dir);
            // make_tbn (utils.h:45-55) with glm's normalize and cross
            F3 t = std::fabs(dir.x) > std::fabs(dir.y) ? F3{-dir.z, 0.0f, dir.x} : F3{0.0f, dir.z, -dir.y};
            t = normf(t);
            const F3 b = crossf(dir, t);
            out.tangent = f4(t);
            out.bitangent = f4(b);
        } else {
            return; // unsupported light type: skipped, as the reference warns and skips
        }
        s.lights.push_back(out);
    }

    bool node(int64_t ni, const M4 &parent, int depth) { // scene.cpp:183-204
        if (depth > 64) {
            err = "node hierarchy too deep (a cycle?)";
            return false;
        }
        const Json &n = d.j["nodes"][(size_t)ni];
        if (n.kind != Json::Object) {
            err = "node " + std::to_string(ni) + " missing";
            return false;
        }
        const M4 g = mulm(parent, node_matrix(n));
        if (n.has("camera"))
            camera(d.j["cameras"][(size_t)n["camera"].integer(0)], g);
        const Json &lref = n["extensions"]["KHR_lights_punctual"]["light"];
        if (lref.kind == Json::Number)
            light(d.j["extensions"]["KHR_lights_punctual"]["lights"][(size_t)lref.integer(0)], g);
        if (n.has("mesh")) {
            const Json &m = d.j["meshes"][(size_t)n["mesh"].integer(0)];
            for (size_t k = 0; k < m["primitives"].size(); k++)
                if (!primitive(m["primitives"][k], g))
                    return false;
        }
        for (size_t k = 0; k < n["children"].size(); k++)
            if (!node(n["children"][k].integer(-1), g, depth + 1))
                return false;
        return true;
    }
};

bool parse_document(const std::string &path, Doc &d, std::string &err) {
    std::vector<uint8_t> raw;
    if (!read_file(path, raw)) {
        err = "cannot read " + path;
        return false;
    }
    const size_t slash = path.find_last_of('/');
    d.dir = slash == std::string::npos ? "." : path.substr(0, slash);
    std::string text;
    std::vector<uint8_t> bin;
    if (raw.size() >= 12 && std::memcmp(raw.data(), "glTF", 4) == 0) { // binary container
        uint32_t hdr[3];
        std::memcpy(hdr, raw.data(), 12);
        if (hdr[1] != 2 || hdr[2] > raw.size()) {
            err = "unsupported .glb version or length";
            return false;
        }
        size_t pos = 12;
        while (pos + 8 <= hdr[2]) {
            uint32_t len, type;
            std::memcpy(&len, raw.data() + pos, 4);
            std::memcpy(&type, raw.data() + pos + 4, 4);
            if (pos + 8 + (size_t)len > hdr[2]) {
                err = "truncated .glb chunk";
                return false;
            }
            if (type == 0x4E4F534Au) // JSON
                text.assign((const char *)raw.data() + pos + 8, len);
            else if (type == 0x004E4942u) // BIN
                bin.assign(raw.data() + pos + 8, raw.data() + pos + 8 + len);
            pos += 8 + (size_t)len;
        }
    } else {
        text.assign(raw.begin(), raw.end());
    }
    try {
        d.j = JsonParser(text).parse();
    } catch (const std::exception &e) {
        err = e.what();
        return false;
    }
    if (d.j["asset"]["version"].string().rfind("2", 0) != 0) {
        err = "not a glTF 2.0 document";
        return false;
    }
    for (size_t i = 0; i < d.j["buffers"].size(); i++) {
        const Json &b = d.j["buffers"][i];
        std::vector<uint8_t> bytes;
        if (b.has("uri")) {
            if (!d.uri_bytes(b["uri"].string(), bytes)) {
                err = "cannot read buffer " + std::to_string(i);
                return false;
            }
        } else {
            bytes = bin;
        }
        d.buffers.push_back(std::move(bytes));
    }
    return true;
}

} // namespace

int scene_load_gltf(const char *path, const phx_gltf_options &opt, SceneStore &s, std::string &err) {
    s = SceneStore{};
    Doc d;
    if (!parse_document(path, d, err))
        return PHX_E_INVALID;
    Loader L(d, s);
    L.load_textures();
    const int64_t sc = d.j["scene"].integer(0);
    const Json &roots = d.j["scenes"][(size_t)sc]["nodes"];
    for (size_t i = 0; i < roots.size(); i++)
        if (!L.node(roots[i].integer(-1), ident(), 0)) {
            err = L.err;
            return PHX_E_INVALID;
        }
    if (s.tris.empty()) {
        err = "the scene has no triangles";
        return PHX_E_INVALID;
    }
    if (L.cams_pos.empty() || opt.camera >= L.cams_pos.size()) {
        err = "the scene has no camera " + std::to_string(opt.camera);
        return PHX_E_INVALID;
    }
    const uint32_t c = opt.camera;
    const float hfov = L.cams_hfov[c];
    if (!(hfov > 0.0f && hfov < 180.0f) || !(L.cams_aspect[c] > 0.0f)) { // scene.cpp:143-146
        err = "camera field of view must lie in (0, 180) degrees and its aspect ratio be positive";
        return PHX_E_INVALID;
    }
    const float aspect = (opt.width && opt.height) ? (float)opt.width / (float)opt.height : L.cams_aspect[c];
    const float P[3] = {L.cams_pos[c].x, L.cams_pos[c].y, L.cams_pos[c].z};
    const float A[3] = {L.cams_at[c].x, L.cams_at[c].y, L.cams_at[c].z};
    const float U[3] = {L.cams_up[c].x, L.cams_up[c].y, L.cams_up[c].z};
    camera_make(P, A, U, hfov, aspect, opt.defocus_angle, opt.focus_distance > 0.0f ? opt.focus_distance : 1.0f,
                &s.camera);
    s.lum.resize(s.lights.size());
    lum_pref_sum(s.lights.data(), (uint32_t)s.lights.size(), s.lum.data());
    return PHX_OK;
}

} // namespace phx
