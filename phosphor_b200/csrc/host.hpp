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

// Device packing of a traversal BVH (see dev_scene.cuh).
struct PackedBvh {
    std::vector<float> cnodes;      // 16 floats per inner node (child pair)
    std::vector<float> wnodes;      // 28 floats per 4-wide node (bvh_widen)
    int32_t wroot = 0;
    uint32_t wdepth = 0;
    std::vector<float> trirec;      // 12 floats per triangle, device (leaf) order
    std::vector<uint32_t> leaf_tri; // device triangle index -> original triangle index
    int32_t root = 0;
    uint32_t max_leaf = 1;
    uint32_t depth = 0;
};
// Leaf rank of every triangle in the reference tree (pre-order over leaves): the tie-break key of
// hits at exactly equal t (hit.h:68 keeps the last tested one).
std::vector<uint32_t> reference_leaf_ranks(const std::vector<phx_bvh_node> &nodes, uint32_t n_tris);
// The reference tree itself re-packed as child pairs (one triangle per leaf).
void bvh_pack(const std::vector<phx_bvh_node> &nodes, const phx_triangle *tris, PackedBvh &out);
// A binned-SAH tree over the same expanded triangle boxes (bounding_box.h:48-61), leaves of up to
// max_leaf triangles; triangle records carry the reference leaf rank for tie-breaking.
bool bvh_build_sah(const phx_triangle *tris, uint32_t n, const std::vector<uint32_t> &ref_rank, uint32_t max_leaf,
                   PackedBvh &out);

// Collapses the child-pair tree into 4-wide nodes (each node pulls up the grandchildren of its
// largest inner children until it has 4): 7 float4 per node, SoA {minx[4], maxx[4], miny[4],
// maxy[4], minz[4], maxz[4], refs[4]}; an empty slot has reference 0x7fffffff (which traversal
// checks: its inverted box would not by itself make the slab test miss).
void bvh_widen(PackedBvh &pk);
// The 4-wide nodes with 8-bit child boxes (bvh_quant.hpp), 16 words per node.
std::vector<uint32_t> bvh_quantize(const PackedBvh &pk);

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

// read_gltf_scene (src/parsers/scene.cpp:206-233) over a glTF 2.0 document (gltf.cpp)
int scene_load_gltf(const char *path, const phx_gltf_options &opt, SceneStore &out, std::string &err);

// Camera::Camera + focus + to_params (src/renderer/camera.cpp:3-56)
int camera_make(const float pos[3], const float at[3], const float up[3], float hfov, float aspect, float defocus,
                float focus, phx_camera_params *out);
// SceneData::build_lum_pref_sum (src/renderer/scene_data.cpp:14-23)
void lum_pref_sum(const phx_light *lights, uint32_t n, float *out);

} // namespace phx
