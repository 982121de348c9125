// ref_host.cpp — TEST INFRASTRUCTURE ONLY.  C entry points over the reference's own host code,
// compiled for the CPU by oracle/build_ref_sppm.py: its BVH builder (src/renderer/bvh.cpp) and
// camera (src/renderer/camera.cpp) and light constructors (src/renderer/light.cpp) are compiled from the reference sources where they lie; the
// photon-grid set-up is the host half of include/common/photon_hash.h; and three functions that
// sit inside classes needing OpenCL or image libraries are read out of their files by the recipe
// into oracle/_ref/host_extract.inc — output.cpp's tone_map/apply_tonemap, shading.cpp's scene
// sphere and scene_data.cpp's light luminance prefix sum.  The reference's host headers are
// compiled against the stand-ins in oracle/ref_shim/ (OpenCL host types, glm, logging).
// Nothing here is product code; the CUDA library never links it.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <execution>
#include <numeric>
#include <stdexcept>
#include <vector>

#include "common/bvh_node.h"
#include "common/constants.h"
#include "common/light.h"
#include "common/photon_hash.h"
#include "common/triangle.h"
#include "host/bvh.hpp"
#include "host/camera.hpp"
#include "host/light.hpp"

#include "host_extract.inc"

#include "../include/phx.h"

static_assert(sizeof(Triangle) == sizeof(phx_triangle) && sizeof(BvhNode) == sizeof(phx_bvh_node) &&
                  sizeof(Light) == sizeof(phx_light) && sizeof(CameraParams) == sizeof(phx_camera_params) &&
                  sizeof(PhotonHashData) == sizeof(phx_photon_hash_data),
              "reference host layouts");

extern "C" {

#define REF_API __attribute__((visibility("default")))

// Bvh::Bvh (bvh.cpp:74-84): 2n-1 nodes.  Returns 1 where the reference would stop with LOG_FATAL
// (a triangle box with an infinity or no width, bounding_box.h:17-28).
REF_API int ref_bvh_build(const phx_triangle *tris, uint32_t n, phx_bvh_node *out) {
    try {
        std::vector<Triangle> t(n);
        std::memcpy(t.data(), tris, (size_t)n * sizeof(Triangle));
        Bvh bvh(t);
        std::memcpy(out, bvh.nodes.data(), bvh.nodes.size() * sizeof(BvhNode));
        return 0;
    } catch (const std::exception &) {
        return 1;
    }
}

// build_photon_hash_info (photon_hash.h:41-50) over the tree's root box, as Renderer::set_scene
// does (renderer.cpp:33-46).
REF_API void ref_hash_info(const phx_bvh_node *root, uint32_t grid_res, phx_photon_hash_data *out) {
    BvhNode node;
    std::memcpy(&node, root, sizeof(node));
    PhotonHashData d = build_photon_hash_info(node.bbox, grid_res);
    std::memcpy(out, &d, sizeof(d));
}

// ShadingBuffers::upload's scene centre and radius (shading.cpp:45-58).
REF_API void ref_scene_sphere(const phx_bvh_node *root, float *center3, float *radius) {
    BvhNode node;
    std::memcpy(&node, root, sizeof(node));
    RefShadingSphere s;
    s.compute(node.bbox);
    center3[0] = s.scene_center.x;
    center3[1] = s.scene_center.y;
    center3[2] = s.scene_center.z;
    *radius = s.scene_radius;
}

// Camera(position, look_at, up, hfov, aspect), then Renderer::set_scene's aspect override and
// focus() (renderer.cpp:25-28), then to_params (camera.cpp:3-56).
REF_API void ref_camera(const float *pos, const float *at, const float *up, float hfov, float aspect,
                        float render_aspect, float defocus_angle, float focus_distance, phx_camera_params *out) {
    Camera cam(vec3(pos[0], pos[1], pos[2]), vec3(at[0], at[1], at[2]), vec3(up[0], up[1], up[2]), hfov, aspect);
    cam.aspect_ratio = render_aspect;
    cam.focus(defocus_angle, focus_distance);
    CameraParams p = cam.to_params();
    std::memcpy(out, &p, sizeof(p));
}

// SceneData::build_lum_pref_sum (scene_data.cpp:14-23).
REF_API void ref_lum_pref_sum(const phx_light *lights, uint32_t n, float *out) {
    RefSceneLum s;
    s.lights.resize(n);
    std::memcpy(s.lights.data(), lights, (size_t)n * sizeof(Light));
    s.build_lum_pref_sum();
    std::copy(s.lum_pref_sum.begin(), s.lum_pref_sum.end(), out);
}

// apply_tonemap (output.cpp:52-83): the 8-bit image of a snapshot.
REF_API void ref_tonemap(uint32_t w, uint32_t h, float exposure, int tonemap, const float *flux4,
                         const float *radiance4, uint64_t total_photons, uint32_t rounds, uint8_t *out) {
    const size_t n = (size_t)w * h;
    std::vector<float4> flux(n), rad(n);
    std::memcpy(flux.data(), flux4, n * sizeof(float4));
    std::memcpy(rad.data(), radiance4, n * sizeof(float4));
    std::vector<u8> ldr = apply_tonemap(w, h, exposure, tonemap != 0, flux, rad, total_photons, rounds);
    std::memcpy(out, ldr.data(), ldr.size());
}

// make_point_light / make_spot_light / make_directional_light / make_textured_light
// (light.cpp:4-45).  kind: 0 point (pos, power), 1 spot (pos, power, dir, a = inner, b = outer
// angle), 2 directional (dir, power), 3 textured (tex, start, count, power, a = total area).
REF_API void ref_make_light(int kind, const float *pos, const float *power, const float *dir, float a, float b,
                            uint32_t tex, uint32_t start, uint32_t count, phx_light *out) {
    vec3 P = pos ? vec3(pos[0], pos[1], pos[2]) : vec3(0.0f), W(power[0], power[1], power[2]);
    vec3 D = dir ? vec3(dir[0], dir[1], dir[2]) : vec3(0.0f);
    Light l = kind == 0   ? make_point_light(P, W)
              : kind == 1 ? make_spot_light(P, W, D, a, b)
              : kind == 2 ? make_directional_light(D, W)
                          : make_textured_light(tex, start, count, W, a);
    std::memcpy(out, &l, sizeof(l));
}

} // extern "C"
