// main.cpp — phx_render: the reference's command line (src/main.cpp:12-61) over libphx.so,
// rendering a glTF 2.0 scene (-m) or one of the procedural scenes.
#include <chrono>
#include <cstdio>
#include <iostream>
#include <memory>

#include "renderer.hpp"

using namespace phx::host;

int main(int argc, char **argv) {
    ArgsList args;
    try {
        args = parse_args(argc, argv);
    } catch (const std::exception &e) {
        if (std::string(e.what()) != "help")
            std::cerr << "error: " << e.what() << "\n";
        std::cerr << usage();
        return 1;
    }
    try {
        int kind = args.scene == "cornell" ? PHX_SCENE_CORNELL : args.scene == "caustic" ? PHX_SCENE_CAUSTIC
                                                                                           : PHX_SCENE_ATRIUM;
        std::unique_ptr<SceneData> owned =
            args.model.empty() ? std::make_unique<SceneData>(kind, args.seed, args.width, args.height, args.scene_detail)
                               : std::make_unique<SceneData>(args.model, args);
        const SceneData &scene = *owned;
        Renderer renderer(args, args.output_dir);
        auto t0 = std::chrono::steady_clock::now();
        renderer.set_scene(scene);
        auto t1 = std::chrono::steady_clock::now();
        uint32_t rounds = renderer.run();
        auto t2 = std::chrono::steady_clock::now();
        phx_info info = renderer.info();
        double setup = std::chrono::duration<double>(t1 - t0).count();
        double render = std::chrono::duration<double>(t2 - t1).count();
        std::printf("%s: %u triangles, %ux%u px, %u rounds x %u photons in %.3fs (set_scene %.3fs): %.2f Mphotons/s, "
                    "%u photons stored last round\n",
                    args.model.empty() ? args.scene.c_str() : args.model.c_str(), scene.scene().n_triangles, info.width, info.height, rounds,
                    info.photons_per_round, render, setup,
                    rounds ? (double)rounds * info.photons_per_round / render / 1e6 : 0.0, info.n_photons);
    } catch (const Error &e) {
        std::cerr << "error (status " << e.code << "): " << e.what() << "\n";
        return 1;
    } catch (const std::exception &e) {
        std::cerr << "error: " << e.what() << "\n";
        return 1;
    }
    return 0;
}
