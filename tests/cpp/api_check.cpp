// A C++ caller of the library's C++ API (include/semper/pipeline.hpp,
// incremental.hpp), for tests/test_gpu_cxx_api.py. Reads raw gray frames,
// writes each call's return code and packed points as raw little-endian
// int32 + float32 records:  [rc, n_floats, floats...] per call.
//
//   api_check full <W> <H> <ref> <def> <mask> <mw> <mh> <mstride> <x y w h step subset window> <out>
//     ReferenceCache::set_from_gray(ref, mask), run_full_field twice (the
//     process-wide token, then a caller's token), then once more with the
//     caller's token requested inside an open CancelScope (expect kCancelled).
//   api_check inc <W> <H> <ref> <x y w h step subset window> <interval> <out> <frame>...
//     IncrementalSession::init, process_frame per frame.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <semper/incremental.hpp>
#include <semper/pipeline.hpp>

using namespace Semper::pipeline;

static std::vector<uint8_t> slurp(const char* path, size_t n) {
    std::vector<uint8_t> v(n);
    FILE* f = std::fopen(path, "rb");
    if (!f || std::fread(v.data(), 1, n, f) != n) std::exit(2);
    std::fclose(f);
    return v;
}

static void record(FILE* f, int rc, const std::vector<float>& out) {
    const int n = rc > 0 ? rc * 8 : 0;
    std::fwrite(&rc, 4, 1, f);
    std::fwrite(&n, 4, 1, f);
    if (n) std::fwrite(out.data(), 4, (size_t)n, f);
}

static FullFieldParams params_from(char** a) {
    FullFieldParams p;
    p.rect_x = std::atoi(a[0]);
    p.rect_y = std::atoi(a[1]);
    p.rect_w = std::atoi(a[2]);
    p.rect_h = std::atoi(a[3]);
    p.step = std::atoi(a[4]);
    p.subset_size = std::atoi(a[5]);
    p.strain_window = std::atoi(a[6]);
    return p;
}

int main(int argc, char** argv) {
    if (argc >= 2 && !std::strcmp(argv[1], "full") && argc == 18) {
        const int W = std::atoi(argv[2]), H = std::atoi(argv[3]);
        const std::vector<uint8_t> ref = slurp(argv[4], (size_t)W * H), def = slurp(argv[5], (size_t)W * H);
        const int mw = std::atoi(argv[7]), mh = std::atoi(argv[8]), ms = std::atoi(argv[9]);
        const std::vector<uint8_t> mask = slurp(argv[6], (size_t)ms * mh);
        const FullFieldParams p = params_from(argv + 10);
        FILE* f = std::fopen(argv[17], "wb");
        if (!f) return 3;
        GrayView rv{ref.data(), W, H, 0}, dv{def.data(), W, H, 0}, mv{mask.data(), mw, mh, (size_t)ms};
        ReferenceCache cache;
        cache.set_from_gray(rv, mv);
        const int cap = (p.rect_w / p.step) * (p.rect_h / p.step) * 8;
        std::vector<float> out((size_t)cap), met(24);
        int last = -1;
        int rc = run_full_field(cache, dv, mv, p, out.data(), cap, met.data(), 24,
                                [&last](int pct) { last = pct; });
        record(f, rc, out);
        CancelToken tok;
        rc = run_full_field(cache, dv, mv, p, out.data(), cap, met.data(), 24, tok);
        record(f, rc, out);
        {
            CancelScope scope(tok);
            tok.request();
            rc = run_full_field(cache, dv, mv, p, out.data(), cap, met.data(), 24, tok);
        }
        record(f, rc, std::vector<float>());
        std::fclose(f);
        std::printf("progress %d\n", last);
        return 0;
    }
    if (argc >= 14 && !std::strcmp(argv[1], "inc")) {
        const int W = std::atoi(argv[2]), H = std::atoi(argv[3]);
        const std::vector<uint8_t> ref = slurp(argv[4], (size_t)W * H);
        IncrementalParams ip;
        ip.field = params_from(argv + 5);
        ip.update_interval = std::atoi(argv[12]);
        FILE* f = std::fopen(argv[13], "wb");
        if (!f) return 3;
        IncrementalSession s;
        if (s.init(GrayView{ref.data(), W, H, 0}, GrayView(), ip) != 0) return 4;
        const int cap = s.max_points() * 8;
        std::vector<float> out((size_t)cap), met(24);
        for (int k = 14; k < argc; ++k) {
            const std::vector<uint8_t> fr = slurp(argv[k], (size_t)W * H);
            IncrementalFrameInfo info;
            const int rc = s.process_frame(GrayView{fr.data(), W, H, 0}, out.data(), cap, met.data(), 24, nullptr,
                                           &info);
            record(f, rc, out);
        }
        std::fclose(f);
        std::printf("frames %d max_points %d\n", s.frames_processed(), s.max_points());
        return 0;
    }
    return 1;
}
