// The boundary's raw-image conversions (csrc/host/gray.hpp) on the CPU, for
// tests/test_boundary.py: reads raw buffers, writes the converted ones.
//   gray_check luma <rgba file> <pixels> <out file>
//   gray_check resize <src file> <sw> <sh> <stride> <dw> <dh> <out file>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "gray.hpp"

static std::vector<uint8_t> slurp(const char* path, size_t n) {
    std::vector<uint8_t> v(n);
    FILE* f = std::fopen(path, "rb");
    if (!f || std::fread(v.data(), 1, n, f) != n) std::exit(2);
    std::fclose(f);
    return v;
}

static void spill(const char* path, const std::vector<uint8_t>& v) {
    FILE* f = std::fopen(path, "wb");
    if (!f || std::fwrite(v.data(), 1, v.size(), f) != v.size()) std::exit(3);
    std::fclose(f);
}

int main(int argc, char** argv) {
    if (argc == 5 && !std::strcmp(argv[1], "luma")) {
        const size_t px = std::strtoul(argv[3], nullptr, 10);
        const std::vector<uint8_t> rgba = slurp(argv[2], 4 * px);
        std::vector<uint8_t> gray(px);
        semper_b200::rgba_to_gray(rgba.data(), px, gray.data());
        spill(argv[4], gray);
        return 0;
    }
    if (argc == 9 && !std::strcmp(argv[1], "resize")) {
        const int sw = std::atoi(argv[3]), sh = std::atoi(argv[4]);
        const size_t stride = std::strtoul(argv[5], nullptr, 10);
        const int dw = std::atoi(argv[6]), dh = std::atoi(argv[7]);
        const std::vector<uint8_t> src = slurp(argv[2], stride * (size_t)sh);
        std::vector<uint8_t> out;
        semper_b200::resize_nearest(src.data(), sw, sh, stride, dw, dh, out);
        spill(argv[8], out);
        return 0;
    }
    return 1;
}
