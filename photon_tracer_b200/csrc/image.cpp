// Image output: write_image and to_display (include/image_write.hpp:15-33,
// include/renderer.hpp:421-423). A path ending in .pfm gets the linear floats
// as a Portable Float Map (header "PF", width height, -1.0 for
// little-endian, rows bottom first); anything else a binary PPM (P6) of
// display bytes, 256 * clamp(sqrt(linear), 0, 0.999) truncated (gamma 2).
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "pt_host.hpp"

extern "C" {

uint8_t pt_to_display(float linear) {
    float s = std::sqrt(linear);
    // clamp (include/vec3.hpp:130-134), in float
    if (s < 0.0f) s = 0.0f;
    if (s > 0.999f) s = 0.999f;
    return static_cast<uint8_t>(256 * s);
}

pt_status pt_write_image(const char* path, int width, int height, const float* linear) {
    pt::clear_error();
    if (!path || !linear || width <= 0 || height <= 0) return pt::fail(PT_ERR_INVALID_ARG, "pt_write_image: bad argument");
    FILE* f = std::fopen(path, "wb");
    if (!f) return pt::fail(PT_ERR_INVALID_ARG, std::string("pt_write_image: cannot open ") + path);
    const std::string p(path);
    const bool pfm = p.size() >= 4 && p.compare(p.size() - 4, 4, ".pfm") == 0;
    bool ok = true;
    const size_t n = 3 * size_t(width) * size_t(height);
    if (pfm) {
        ok = std::fprintf(f, "PF\n%d %d\n-1.0\n", width, height) > 0;
        for (int y = height - 1; y >= 0 && ok; --y)
            ok = std::fwrite(linear + 3 * size_t(y) * width, sizeof(float), 3 * size_t(width), f) == 3 * size_t(width);
    } else {
        std::vector<uint8_t> bytes(n);
        for (size_t c = 0; c < n; ++c) bytes[c] = pt_to_display(linear[c]);
        ok = std::fprintf(f, "P6\n%d %d\n255\n", width, height) > 0 && std::fwrite(bytes.data(), 1, n, f) == n;
    }
    ok = (std::fclose(f) == 0) && ok;
    return ok ? PT_OK : pt::fail(PT_ERR_INVALID_ARG, std::string("pt_write_image: failed to write ") + path);
}

}  // extern "C"
