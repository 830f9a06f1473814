// render_scene: renders a serialized scene file through the C++ mirror (include/htcuda.hpp)
// and writes the RGBA8 result.
//
//   render_scene <scene.bin> <recipe 1|2> <hops> <width> <height> <passes> <seeds.u32> <out.rgba>
//
// scene.bin holds the bytes the reference's serializer writes; seeds.u32 one uint32 per pixel.
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iterator>
#include <vector>

#include "../../../include/htcuda.hpp"

static std::vector<uint8_t> read_file(const char *path) {
    std::ifstream f(path, std::ios::binary);
    return std::vector<uint8_t>(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
}

int main(int argc, char **argv) {
    if (argc != 9) {
        std::fprintf(stderr, "usage: %s scene.bin recipe hops width height passes seeds.u32 out.rgba\n", argv[0]);
        return 2;
    }
    try {
        const auto scene = read_file(argv[1]);
        const int recipe = std::atoi(argv[2]);
        const uint32_t hops = (uint32_t)std::atoi(argv[3]);
        const uint32_t w = (uint32_t)std::atoi(argv[4]), h = (uint32_t)std::atoi(argv[5]);
        const uint32_t passes = (uint32_t)std::atoi(argv[6]);
        const auto seed_bytes = read_file(argv[7]);
        std::vector<uint32_t> seeds(seed_bytes.size() / 4);
        std::memcpy(seeds.data(), seed_bytes.data(), seeds.size() * 4);
        htc::Context ctx(0);
        htc::Pipeline pipe(ctx, w, h, recipe, hops, scene, seeds);
        pipe.render(passes);
        const auto img = pipe.get_image();
        std::ofstream out(argv[8], std::ios::binary);
        out.write(reinterpret_cast<const char *>(img.data()), (std::streamsize)img.size());
        return 0;
    } catch (const htc::Error &e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
}
