// renderer.cpp — C++ host API over the C ABI (see renderer.hpp).
#include "renderer.hpp"

#include <cstring>
#include <fstream>
#include <sstream>

namespace phx::host {

void check(int status) {
    if (status != PHX_OK)
        throw Error(status, phx_last_error());
}

phx_params ArgsList::params() const {
    phx_params p{};
    p.width = width;
    p.height = height;
    p.photons_per_round = photons_per_round;
    p.max_photon_bounces = max_photon_bounces;
    p.grid_res = grid_res;
    p.sppm_alpha = sppm_alpha;
    p.direct_samples = direct_samples;
    p.seed = seed;
    p.flags = 0;
    return p;
}

std::string usage() {
    return "usage: phx_render [flags]\n"
           "  -w <px> -h <px>          image size (1024 x 1024)\n"
           "  --exposure <f>           colour exposure multiplier (0.66)\n"
           "  --tonemap                apply ACES tone mapping\n"
           "  --seed <u32>             seed of the round RNG (2137)\n"
           "  -p <u32>                 photons emitted per SPPM round (2^20)\n"
           "  --max-bounces <1..32>    max photon bounces (16)\n"
           "  --grid-res <1..255>      resolution of the photon hash grid (64)\n"
           "  --defocus-angle <deg>    (0)   --focus-distance <f> (1)\n"
           "  --sppm-rounds <u32>      number of SPPM rounds (64)\n"
           "  --sppm-alpha <f>         radius reduction ratio (0.7)\n"
           "  --direct-samples <1..128> direct-lighting samples per pixel per round (16)\n"
           "  -m <file.glb|file.gltf>  glTF 2.0 scene to render\n"
           "  --scene <cornell|caustic|atrium> [--detail n]   procedural scene (when no -m is given)\n"
           "  -o <dir>                 output directory\n"
           "  --snapshots              also write images at power-of-two rounds\n"
           "  --plain                  per-pass launches with host syncs (default: graph replay)\n"
           "  --device <n>             CUDA device\n"
           "  --batch-size, --workgroup, --ray-step are accepted for compatibility and ignored\n";
}

ArgsList parse_args(int argc, char **argv) {
    ArgsList a;
    auto need = [&](int &i) -> std::string {
        if (i + 1 >= argc)
            throw std::invalid_argument(std::string("missing value for ") + argv[i]);
        return argv[++i];
    };
    auto u32v = [](const std::string &s, uint32_t lo, uint32_t hi, const char *name) {
        unsigned long v = std::stoul(s);
        if (v < lo || v > hi)
            throw std::invalid_argument(std::string(name) + " out of range");
        return (uint32_t)v;
    };
    auto f32v = [](const std::string &s, const char *name) {
        float v = std::stof(s);
        if (!(v >= 0.0f))
            throw std::invalid_argument(std::string(name) + " must be non-negative");
        return v;
    };
    for (int i = 1; i < argc; i++) {
        std::string f = argv[i];
        if (f == "--help")
            throw std::invalid_argument("help");
        else if (f == "-w")
            a.width = u32v(need(i), 1, 1u << 15, "-w");
        else if (f == "-h")
            a.height = u32v(need(i), 1, 1u << 15, "-h");
        else if (f == "--exposure")
            a.exposure = f32v(need(i), "--exposure");
        else if (f == "--tonemap")
            a.tonemap = true;
        else if (f == "--batch-size")
            a.max_photons_per_batch = u32v(need(i), 1, 0xffffffffu, "--batch-size");
        else if (f == "--workgroup")
            a.workgroup_size = u32v(need(i), 1, 1024, "--workgroup");
        else if (f == "--seed")
            a.seed = u32v(need(i), 0, 0xffffffffu, "--seed");
        else if (f == "-p")
            a.photons_per_round = u32v(need(i), 1, 0xffffffffu, "-p");
        else if (f == "--ray-step")
            a.ray_step = f32v(need(i), "--ray-step");
        else if (f == "--max-bounces")
            a.max_photon_bounces = u32v(need(i), 1, 32, "--max-bounces");
        else if (f == "--grid-res")
            a.grid_res = u32v(need(i), 1, 255, "--grid-res");
        else if (f == "--defocus-angle")
            a.defocus_angle = f32v(need(i), "--defocus-angle");
        else if (f == "--focus-distance")
            a.focus_distance = f32v(need(i), "--focus-distance");
        else if (f == "--sppm-rounds")
            a.sppm_rounds = u32v(need(i), 0, 0xffffffffu, "--sppm-rounds");
        else if (f == "--sppm-alpha")
            a.sppm_alpha = f32v(need(i), "--sppm-alpha");
        else if (f == "--direct-samples")
            a.direct_samples = u32v(need(i), 1, 128, "--direct-samples");
        else if (f == "-m")
            a.model = need(i);
        else if (f == "--scene")
            a.scene = need(i);
        else if (f == "--detail")
            a.scene_detail = u32v(need(i), 0, 4096, "--detail");
        else if (f == "-o")
            a.output_dir = need(i);
        else if (f == "--snapshots")
            a.save_snapshots = true;
        else if (f == "--plain")
            a.graph = false;
        else if (f == "--device")
            a.device = (int)u32v(need(i), 0, 64, "--device");
        else
            throw std::invalid_argument("unknown flag " + f);
    }
    if (a.scene != "cornell" && a.scene != "caustic" && a.scene != "atrium")
        throw std::invalid_argument("--scene must be cornell, caustic or atrium");
    return a;
}

SceneData::SceneData(int kind, uint32_t seed, uint32_t width, uint32_t height, uint32_t detail) {
    phx_scene_spec spec{};
    spec.kind = kind;
    spec.seed = seed;
    spec.width = width;
    spec.height = height;
    spec.detail = detail;
    check(phx_scene_generate(&spec, &scene_, &handle_));
}

SceneData::SceneData(const std::string &gltf_path, const ArgsList &args) {
    phx_gltf_options opt{};
    opt.width = args.width;
    opt.height = args.height;
    opt.defocus_angle = args.defocus_angle;
    opt.focus_distance = args.focus_distance;
    check(phx_scene_load_gltf(gltf_path.c_str(), &opt, &scene_, &handle_));
}

SceneData::~SceneData() {
    if (handle_)
        phx_scene_free(handle_);
}

// ---- PNG --------------------------------------------------------------------------------------
namespace {
uint32_t crc32(const uint8_t *p, size_t n, uint32_t c = 0xffffffffu) {
    static uint32_t table[256];
    static bool init = false;
    if (!init) {
        for (uint32_t i = 0; i < 256; i++) {
            uint32_t x = i;
            for (int k = 0; k < 8; k++)
                x = (x & 1) ? 0xedb88320u ^ (x >> 1) : x >> 1;
            table[i] = x;
        }
        init = true;
    }
    for (size_t i = 0; i < n; i++)
        c = table[(c ^ p[i]) & 0xff] ^ (c >> 8);
    return c;
}
void be32(std::vector<uint8_t> &o, uint32_t v) {
    for (int s = 24; s >= 0; s -= 8)
        o.push_back((uint8_t)(v >> s));
}
void chunk(std::vector<uint8_t> &o, const char *tag, const std::vector<uint8_t> &data) {
    be32(o, (uint32_t)data.size());
    size_t start = o.size();
    o.insert(o.end(), tag, tag + 4);
    o.insert(o.end(), data.begin(), data.end());
    be32(o, crc32(o.data() + start, o.size() - start) ^ 0xffffffffu);
}
} // namespace

std::vector<uint8_t> encode_png(const uint8_t *rgb, uint32_t w, uint32_t h) {
    std::vector<uint8_t> raw;
    raw.reserve((size_t)h * (3 * w + 1));
    for (uint32_t y = 0; y < h; y++) {
        raw.push_back(0);
        raw.insert(raw.end(), rgb + (size_t)y * 3 * w, rgb + (size_t)(y + 1) * 3 * w);
    }
    // zlib stream of stored (uncompressed) deflate blocks
    std::vector<uint8_t> z{0x78, 0x01};
    size_t pos = 0;
    do {
        size_t n = std::min<size_t>(65535, raw.size() - pos);
        bool last = pos + n == raw.size();
        z.push_back(last ? 1 : 0);
        z.push_back((uint8_t)(n & 0xff));
        z.push_back((uint8_t)(n >> 8));
        z.push_back((uint8_t)(~n & 0xff));
        z.push_back((uint8_t)((~n >> 8) & 0xff));
        z.insert(z.end(), raw.begin() + pos, raw.begin() + pos + n);
        pos += n;
    } while (pos < raw.size());
    uint32_t a = 1, b = 0;
    for (uint8_t c : raw) {
        a = (a + c) % 65521;
        b = (b + a) % 65521;
    }
    be32(z, (b << 16) | a);
    std::vector<uint8_t> png{0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n'};
    std::vector<uint8_t> ihdr;
    be32(ihdr, w);
    be32(ihdr, h);
    ihdr.insert(ihdr.end(), {8, 2, 0, 0, 0});
    chunk(png, "IHDR", ihdr);
    chunk(png, "IDAT", z);
    chunk(png, "IEND", {});
    return png;
}

// ---- ImageWriter (output.cpp:100-153) -----------------------------------------------------------
ImageWriter::ImageWriter() : worker_([this] { worker_loop(); }) {}

ImageWriter::~ImageWriter() {
    flush();
    {
        std::lock_guard<std::mutex> lock(mutex_);
        stop_ = true;
    }
    cv_jobs_.notify_one();
    if (worker_.joinable())
        worker_.join();
}

void ImageWriter::submit(const std::filesystem::path &path, uint32_t width, uint32_t height,
                         std::vector<uint8_t> ldr) {
    {
        std::lock_guard<std::mutex> lock(mutex_);
        jobs_.push(Job{path, width, height, std::move(ldr)});
        active_++;
    }
    cv_jobs_.notify_one();
}

void ImageWriter::flush() {
    std::unique_lock<std::mutex> lock(mutex_);
    cv_flush_.wait(lock, [this] { return jobs_.empty() && active_ == 0; });
}

void ImageWriter::worker_loop() {
    for (;;) {
        Job job;
        {
            std::unique_lock<std::mutex> lock(mutex_);
            cv_jobs_.wait(lock, [this] { return !jobs_.empty() || stop_; });
            if (jobs_.empty() && stop_)
                return;
            job = std::move(jobs_.front());
            jobs_.pop();
        }
        std::vector<uint8_t> png = encode_png(job.ldr.data(), job.width, job.height);
        std::ofstream(job.path, std::ios::binary).write((const char *)png.data(), (std::streamsize)png.size());
        {
            std::lock_guard<std::mutex> lock(mutex_);
            active_--;
            if (active_ == 0 && jobs_.empty())
                cv_flush_.notify_all();
        }
    }
}

// ---- Renderer ---------------------------------------------------------------------------------
Renderer::Renderer(ArgsList args, std::filesystem::path output_dir, std::string image_metadata)
    : args_(std::move(args)), output_dir_(std::move(output_dir)), metadata_(std::move(image_metadata)) {}

Renderer::~Renderer() {
    writer_.flush();
    if (ctx_)
        phx_destroy(ctx_);
}

void Renderer::set_scene(const SceneData &scene) {
    if (ctx_) {
        phx_destroy(ctx_);
        ctx_ = nullptr;
    }
    phx_params p = args_.params();
    check(phx_create(&scene.scene(), &p, args_.device, &ctx_));
}

void Renderer::trace_rays(uint32_t seed) { check(phx_trace_rays(ctx_, seed)); }

uint32_t Renderer::emit_photons(uint32_t seed) {
    check(phx_emit_photons(ctx_, seed));
    return info().n_photons;
}

void Renderer::hash_and_sort_photons() { check(phx_hash_sort(ctx_)); }

void Renderer::gather_flux() { check(phx_gather(ctx_, args_.sppm_alpha)); }

phx_info Renderer::info() const {
    phx_info i{};
    check(phx_get_info(ctx_, &i));
    return i;
}

std::vector<uint8_t> Renderer::image_ldr() const {
    phx_info i = info();
    std::vector<uint8_t> ldr((size_t)i.width * i.height * 3);
    check(phx_image(ctx_, args_.exposure, args_.tonemap ? 1 : 0, 0, 0, nullptr, ldr.data()));
    return ldr;
}

std::filesystem::path Renderer::save_snapshot(uint32_t round) {
    std::filesystem::create_directories(output_dir_);
    char name[32];
    std::snprintf(name, sizeof(name), "%06u.png", round);
    std::filesystem::path path = output_dir_ / name;
    phx_info i = info();
    writer_.submit(path, i.width, i.height, image_ldr());
    return path;
}

uint32_t Renderer::run() {
    if (!ctx_)
        throw Error(PHX_E_STATE, "set_scene() first");
    const uint32_t rounds = args_.sppm_rounds;
    uint32_t done = 0;
    while (done < rounds) {
        uint32_t step = rounds - done;
        if (args_.save_snapshots) { // stop at the next power of two (renderer.cpp:79)
            uint32_t next = 1;
            while (next <= done)
                next <<= 1;
            step = std::min(step, next - done);
        }
        if (args_.graph) {
            check(phx_iterate(ctx_, step));
        } else {
            for (uint32_t k = 0; k < step; k++)
                check(phx_round(ctx_));
        }
        done += step;
        bool pow2 = (done & (done - 1)) == 0;
        if ((args_.save_snapshots && pow2) || done == rounds)
            save_snapshot(done);
    }
    writer_.flush();
    return done;
}

} // namespace phx::host
