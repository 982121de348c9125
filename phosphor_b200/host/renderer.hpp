// renderer.hpp — C++ host API of the SPPM core, shaped like the reference's host classes
// (include/host/renderer.hpp:16-72, include/host/output.hpp:14-55, include/host/cmd_args.hpp:11-75).
// It is a pure client of the C ABI (include/phx.h): no CUDA types, no device pointers.
#pragma once

#include <condition_variable>
#include <cstdint>
#include <filesystem>
#include <mutex>
#include <queue>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/phx.h"

namespace phx::host {

// The flags of ARG_TABLE (cmd_args.hpp:36-65) with the reference defaults (cmd_args.hpp:11-34).
struct ArgsList {
    uint32_t width = 1024, height = 1024;
    float exposure = 0.66f;
    bool tonemap = false;
    uint32_t max_photons_per_batch = 1u << 20;
    uint32_t workgroup_size = 32;
    uint32_t seed = 2137;
    uint32_t photons_per_round = 1u << 20;
    float ray_step = 0.0001f; // parsed but unused by the reference (cmd_args.hpp:48)
    uint32_t max_photon_bounces = 16;
    uint32_t grid_res = 64;
    float defocus_angle = 0.0f;
    float focus_distance = 1.0f;
    uint32_t sppm_rounds = 64;
    float sppm_alpha = 0.7f;
    uint32_t direct_samples = 16;
    std::string model;             // -m: a .glb / .gltf scene file (read_gltf_scene)
    std::string scene = "cornell"; // procedural scene when no -m is given
    uint32_t scene_detail = 0;
    std::string output_dir = "./phosphor_output";
    bool save_snapshots = false;
    bool graph = true; // replay rounds from a captured CUDA graph (false: per-pass launches)
    int device = 0;

    phx_params params() const;
};

// Parses the reference's flag vocabulary; throws std::invalid_argument with a message.
ArgsList parse_args(int argc, char **argv);
std::string usage();

class Error : public std::runtime_error {
  public:
    Error(int code, const std::string &msg) : std::runtime_error(msg), code(code) {}
    int code;
};

// Host scene arrays (SceneData, include/host/scene_data.hpp:21-42), from a procedural generator.
class SceneData {
  public:
    SceneData(int kind, uint32_t seed, uint32_t width, uint32_t height, uint32_t detail = 0);
    // a glTF 2.0 file (scene.cpp:206-233) with the render size and focus of `args` (renderer.cpp:24-28)
    SceneData(const std::string &gltf_path, const ArgsList &args);
    ~SceneData();
    SceneData(const SceneData &) = delete;
    SceneData &operator=(const SceneData &) = delete;
    const phx_scene &scene() const { return scene_; }

  private:
    phx_scene scene_{};
    void *handle_ = nullptr;
};

// 8-bit RGB PNG encoder (stored deflate blocks) — the reference uses stb_image_write.
std::vector<uint8_t> encode_png(const uint8_t *rgb, uint32_t width, uint32_t height);

// Asynchronous image writer (output.cpp:100-153): submit() queues an 8-bit image, a worker
// thread writes the PNG; flush() waits for the queue to drain.
class ImageWriter {
  public:
    ImageWriter();
    ~ImageWriter();
    void submit(const std::filesystem::path &path, uint32_t width, uint32_t height, std::vector<uint8_t> ldr);
    void flush();

  private:
    struct Job {
        std::filesystem::path path;
        uint32_t width, height;
        std::vector<uint8_t> ldr;
    };
    void worker_loop();
    std::mutex mutex_;
    std::condition_variable cv_jobs_, cv_flush_;
    std::queue<Job> jobs_;
    uint32_t active_ = 0;
    bool stop_ = false;
    std::thread worker_;
};

// Renderer(args, output_dir, metadata) -> set_scene(scene) -> run() (renderer.cpp:9-169).
class Renderer {
  public:
    Renderer(ArgsList args, std::filesystem::path output_dir, std::string image_metadata = "");
    ~Renderer();
    Renderer(const Renderer &) = delete;
    Renderer &operator=(const Renderer &) = delete;

    void set_scene(const SceneData &scene);
    // runs args.sppm_rounds rounds, writing snapshots at powers of two (when enabled) and the
    // final image; returns the number of rounds run
    uint32_t run();

    // the reference's per-pass stages (private there)
    void trace_rays(uint32_t seed);
    uint32_t emit_photons(uint32_t seed);
    void hash_and_sort_photons();
    void gather_flux();

    phx_info info() const;
    std::vector<uint8_t> image_ldr() const;
    std::filesystem::path save_snapshot(uint32_t round);
    void *context() const { return ctx_; }

  private:
    ArgsList args_;
    std::filesystem::path output_dir_;
    std::string metadata_;
    void *ctx_ = nullptr;
    ImageWriter writer_;
};

void check(int status);

} // namespace phx::host
