// host.hpp — host-side pieces of the renderer core that run once per scene: BVH construction,
// its device packing, camera basis, light prefix sums and the procedural scene generators.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/phx.h"

namespace phx {

// Bvh::Bvh (src/renderer/bvh.cpp:18-84).  Returns false on a degenerate triangle box
// (bounding_box.h:17-28 traps there).
bool bvh_build(const phx_triangle *tris, uint32_t n, std::vector<phx_bvh_node> &nodes, uint32_t *depth);

// Device packing of a reference-layout BVH (see dev_scene.cuh).
struct PackedBvh {
    std::vector<float> cnodes;     // 16 floats per inner node
    std::vector<float> trirec;     // 12 floats per triangle, leaf order
    std::vector<uint32_t> leaf_tri; // leaf rank -> original triangle index
    int32_t root = 0;
};
void bvh_pack(const std::vector<phx_bvh_node> &nodes, const phx_triangle *tris, PackedBvh &out);

phx_photon_hash_data hash_info(const phx_bvh_node &root, uint32_t grid_res);
void scene_sphere(const phx_bvh_node &root, phx_f4 *center, float *radius);

// Owned storage behind a phx_scene.
struct SceneStore {
    std::vector<phx_triangle> tris, etris;
    std::vector<phx_material> mats;
    std::vector<phx_uv_transform_block> uvs;
    std::vector<phx_light> lights;
    std::vector<float> lum;
    std::vector<phx_texture_meta> tex_meta;
    std::vector<uint8_t> atlas;
    std::vector<float> envmap;
    uint32_t env_w = 0, env_h = 0;
    phx_camera_params camera{};
    void view(phx_scene *out) const;
};

int scene_generate(const phx_scene_spec &spec, SceneStore &out, std::string &err);

// Camera::Camera + focus + to_params (src/renderer/camera.cpp:3-56)
int camera_make(const float pos[3], const float at[3], const float up[3], float hfov, float aspect, float defocus,
                float focus, phx_camera_params *out);
// SceneData::build_lum_pref_sum (src/renderer/scene_data.cpp:14-23)
void lum_pref_sum(const phx_light *lights, uint32_t n, float *out);

} // namespace phx
