// Command-line front end of the B200 BM3D, mirroring the reference's
// `ISP_MW --bm3d [options] input` (source/ISP_MW.cpp:200-290, BM3D_IO in
// include/BM3D.h:362-527, FilterIO in include/Filter.h:220-321) over raw
// files instead of OpenCV images.
//
//   isp_mw --bm3d [options] INPUT
//
// Filter options (BM3D_IO, same spelling):
//   -P, --profile NAME                      fast | lc | np | high | vn (default fast)
//   -S, --sigma V                           repeat up to 3 times (Y, U, V); missing values
//                                           repeat the last; the final stage takes the same
//   -BS1/-BSP1/-GS1/-MR1/-MS1/-TH1 V        basic BlockSize / BlockStep / GroupSize /
//       (--BlockSize1 ... --thMSE1)         BMrange / BMstep / thMSE
//   -LD, --lambda V                         basic lambda
//   -BS2/-BSP2/-GS2/-MR2/-MS2/-TH2 V        the same for the final stage
//   --ref PATH                              reference image (same raw layout as INPUT)
// Output naming (FilterIO): -T, --tag TAG (default ".BM3D"), -F, --format EXT
// (default ".raw"): OUTPUT = INPUT without extension + TAG + EXT.
// Raw layout (replaces the image reader):
//   -W, --width N, -H, --height N           plane size (required)
//   --type rgb | gray | float               rgb: three planar integer planes R, G, B;
//                                           gray: one integer plane; float: one float32
//                                           plane, luma range [0, 1] (default rgb)
//   --depth 8..16                           bits per integer sample (default 8); stored as
//                                           uint8 (8) or little-endian uint16 (9..16)
//   --tv                                    limited range ([16, 235] << (depth - 8))
//   --device N                              CUDA device (default 0)
// Exit status: 0 done, 1 unknown filter (the reference's other filters are not
// part of this build), 2 bad arguments or I/O error, 3 filter error.
#include "bm3d_b200/BM3D.hpp"

#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace {

struct Options {
    std::string input, ref, tag = ".BM3D", format = ".raw", type = "rgb";
    int width = 0, height = 0, depth = 8, device = 0;
    bool tv = false;
};

[[noreturn]] void fail(int code, const std::string &msg)
{
    std::fprintf(stderr, "isp_mw: %s\n", msg.c_str());
    std::exit(code);
}

bool next_value(const std::vector<std::string> &a, size_t &i, std::string &out)
{
    if (i + 1 >= a.size()) return false;
    out = a[++i];
    return true;
}

long to_int(const std::string &s, const std::string &flag)
{
    char *end = nullptr;
    const long v = std::strtol(s.c_str(), &end, 10);
    if (s.empty() || *end) fail(2, "bad integer for " + flag + ": " + s);
    return v;
}

double to_double(const std::string &s, const std::string &flag)
{
    char *end = nullptr;
    const double v = std::strtod(s.c_str(), &end);
    if (s.empty() || *end) fail(2, "bad number for " + flag + ": " + s);
    return v;
}

// BM3D_IO::arguments_process (include/BM3D.h:374-488): a profile pass first,
// then the parameters, then sigma padding and thMSE defaults.
void parse(const std::vector<std::string> &a, Options &o, BM3D_Para &para)
{
    std::string v;
    for (size_t i = 0; i < a.size(); ++i) {
        if (a[i] == "-P" || a[i] == "--profile") {
            if (!next_value(a, i, v)) fail(2, "missing value for " + a[i]);
            try {
                para = BM3D_Para(v);
            } catch (const bm3d_b200::Error &e) {
                fail(2, e.what());
            }
        } else if (a[i].size() > 1 && a[i][0] == '-' && a[i] != "--tv") {
            ++i;
        }
    }
    bool th1 = false, th2 = false;
    std::vector<double> sigma;
    for (size_t i = 0; i < a.size(); ++i) {
        const std::string &f = a[i];
        auto val = [&]() -> std::string {
            std::string s;
            if (!next_value(a, i, s)) fail(2, "missing value for " + f);
            return s;
        };
        auto is = [&](const char *s1, const char *s2) { return f == s1 || f == s2; };
        if (is("-P", "--profile")) { val(); }
        else if (f == "--ref") o.ref = val();
        else if (is("-S", "--sigma")) sigma.push_back(to_double(val(), f));
        else if (is("-BS1", "--BlockSize1")) para.basic.BlockSize = static_cast<int>(to_int(val(), f));
        else if (is("-BSP1", "--BlockStep1")) para.basic.BlockStep = static_cast<int>(to_int(val(), f));
        else if (is("-GS1", "--GroupSize1")) para.basic.GroupSize = static_cast<int>(to_int(val(), f));
        else if (is("-MR1", "--BMrange1")) para.basic.BMrange = static_cast<int>(to_int(val(), f));
        else if (is("-MS1", "--BMstep1")) para.basic.BMstep = static_cast<int>(to_int(val(), f));
        else if (is("-TH1", "--thMSE1")) { para.basic.thMSE = to_double(val(), f); th1 = true; }
        else if (is("-LD", "--lambda")) para.basic.lambda = to_double(val(), f);
        else if (is("-BS2", "--BlockSize2")) para.final.BlockSize = static_cast<int>(to_int(val(), f));
        else if (is("-BSP2", "--BlockStep2")) para.final.BlockStep = static_cast<int>(to_int(val(), f));
        else if (is("-GS2", "--GroupSize2")) para.final.GroupSize = static_cast<int>(to_int(val(), f));
        else if (is("-MR2", "--BMrange2")) para.final.BMrange = static_cast<int>(to_int(val(), f));
        else if (is("-MS2", "--BMstep2")) para.final.BMstep = static_cast<int>(to_int(val(), f));
        else if (is("-TH2", "--thMSE2")) { para.final.thMSE = to_double(val(), f); th2 = true; }
        else if (is("-T", "--tag")) o.tag = val();
        else if (is("-F", "--format")) o.format = val();
        else if (is("-W", "--width")) o.width = static_cast<int>(to_int(val(), f));
        else if (is("-H", "--height")) o.height = static_cast<int>(to_int(val(), f));
        else if (f == "--type") o.type = val();
        else if (f == "--depth") o.depth = static_cast<int>(to_int(val(), f));
        else if (f == "--device") o.device = static_cast<int>(to_int(val(), f));
        else if (f == "--tv") o.tv = true;
        else if (f.size() > 1 && f[0] == '-') fail(2, "unknown option " + f);
        else o.input = f;
    }
    if (!sigma.empty()) {
        while (sigma.size() < 3) sigma.push_back(sigma.back());
        para.basic.sigma = sigma;
    }
    para.final.sigma = para.basic.sigma;
    if (!th1) para.basic.thMSE_Default();
    if (!th2) para.final.thMSE_Default();
}

// FilterIO::generate_OPath (include/Filter.h:235-245): directory and stem of
// the input, then the tag and the format.
std::string output_path(const Options &o)
{
    const size_t slash = o.input.find_last_of("/\\");
    const size_t dot = o.input.find_last_of('.');
    const std::string stem =
        dot != std::string::npos && (slash == std::string::npos || dot > slash) ? o.input.substr(0, dot)
                                                                                  : o.input;
    return stem + o.tag + o.format;
}

std::vector<unsigned char> read_file(const std::string &path, size_t bytes)
{
    std::vector<unsigned char> buf(bytes);
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) fail(2, "cannot open " + path);
    const size_t got = std::fread(buf.data(), 1, bytes, f);
    std::fclose(f);
    if (got != bytes) fail(2, path + ": expected " + std::to_string(bytes) + " bytes");
    return buf;
}

void write_file(const std::string &path, const std::vector<unsigned char> &buf)
{
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f || std::fwrite(buf.data(), 1, buf.size(), f) != buf.size()) fail(2, "cannot write " + path);
    std::fclose(f);
}

// Integer samples <-> bytes: uint8, or little-endian uint16 for depth > 8.
void unpack(const std::vector<unsigned char> &buf, size_t offset, Plane &p, int depth)
{
    const size_t n = static_cast<size_t>(p.PixelCount());
    for (size_t i = 0; i < n; ++i)
        p[static_cast<PCType>(i)] = depth > 8 ? buf[offset + 2 * i] | (buf[offset + 2 * i + 1] << 8)
                                              : buf[offset + i];
}

void pack(std::vector<unsigned char> &buf, size_t offset, const Plane &p, int depth)
{
    const size_t n = static_cast<size_t>(p.PixelCount());
    for (size_t i = 0; i < n; ++i) {
        const int v = p[static_cast<PCType>(i)];
        if (depth > 8) {
            buf[offset + 2 * i] = static_cast<unsigned char>(v & 0xff);
            buf[offset + 2 * i + 1] = static_cast<unsigned char>((v >> 8) & 0xff);
        } else {
            buf[offset + i] = static_cast<unsigned char>(v);
        }
    }
}

int run_bm3d(const std::vector<std::string> &args)
{
    Options o;
    BM3D_Para para("fast");
    parse(args, o, para);
    if (o.input.empty()) fail(2, "no input file");
    if (o.width <= 0 || o.height <= 0) fail(2, "--width and --height are required");
    if (o.depth < 8 || o.depth > 16) fail(2, "--depth must be 8..16");
    if (o.type != "rgb" && o.type != "gray" && o.type != "float") fail(2, "unknown --type " + o.type);
    const std::string out = output_path(o);
    const size_t npx = static_cast<size_t>(o.width) * o.height;
    const size_t sample = o.depth > 8 ? 2 : 1;
    // inputs are read before any device work
    const size_t bytes = o.type == "float" ? npx * 4 : (o.type == "gray" ? 1 : 3) * npx * sample;
    const std::vector<unsigned char> in_buf = read_file(o.input, bytes);
    const std::vector<unsigned char> ref_buf =
        o.ref.empty() ? std::vector<unsigned char>() : read_file(o.ref, bytes);
    bm3d_ctx *ctx = nullptr;
    try {
        if (bm3d_ctx_create(&ctx, o.device) != BM3D_OK)
            throw bm3d_b200::Error(BM3D_ERR_CUDA, bm3d_last_error(nullptr));
        BM3D filter(para, ctx);
        if (o.type == "float") {
            Plane_FL src(0.f, o.width, o.height, true, false, false);
            std::memcpy(src.data(), in_buf.data(), npx * 4);
            Plane_FL dst(src, false);
            if (o.ref.empty()) {
                filter.process(dst, src);
            } else {
                Plane_FL ref(src, false);
                std::memcpy(ref.data(), ref_buf.data(), npx * 4);
                filter.process(dst, src, ref);
            }
            std::vector<unsigned char> ob(npx * 4);
            std::memcpy(ob.data(), dst.data(), npx * 4);
            write_file(out, ob);
        } else if (o.type == "gray") {
            const int lo = o.tv ? 16 << (o.depth - 8) : 0;
            const int hi = o.tv ? 235 << (o.depth - 8) : (1 << o.depth) - 1;
            Plane src(0, o.width, o.height, o.depth, lo, lo, hi, false);
            unpack(in_buf, 0, src, o.depth);
            Plane dst(src, false);
            if (o.ref.empty()) {
                filter.process(dst, src);
            } else {
                Plane ref(src, false);
                unpack(ref_buf, 0, ref, o.depth);
                filter.process(dst, src, ref);
            }
            std::vector<unsigned char> ob(npx * sample);
            pack(ob, 0, dst, o.depth);
            write_file(out, ob);
        } else {
            Frame src(0, o.width, o.height, o.depth, !o.tv);
            for (int c = 0; c < 3; ++c) unpack(in_buf, c * npx * sample, src.P(c), o.depth);
            Frame dst(src, false);
            if (o.ref.empty()) {
                filter.process(dst, src);
            } else {
                Frame ref(src, false);
                for (int c = 0; c < 3; ++c) unpack(ref_buf, c * npx * sample, ref.P(c), o.depth);
                filter.process(dst, src, ref);
            }
            std::vector<unsigned char> ob(3 * npx * sample);
            for (int c = 0; c < 3; ++c) pack(ob, c * npx * sample, dst.P(c), o.depth);
            write_file(out, ob);
        }
    } catch (const bm3d_b200::Error &e) {
        if (ctx) bm3d_ctx_destroy(ctx);
        std::fprintf(stderr, "isp_mw: %s\n", e.what());
        return 3;
    }
    bm3d_ctx_destroy(ctx);
    std::printf("%s\n", out.c_str());
    return 0;
}

}  // namespace

// Filtering (source/ISP_MW.cpp:200-290): the first argument names the filter.
int main(int argc, char **argv)
{
    if (argc <= 2) {
        std::printf("Not enough arguments specified.\n");
        return 0;
    }
    std::string name = argv[1];
    for (auto &ch : name) ch = static_cast<char>(std::tolower(static_cast<unsigned char>(ch)));
    std::vector<std::string> args(argv + 2, argv + argc);
    if (name == "--bm3d") return run_bm3d(args);
    std::fprintf(stderr, "isp_mw: filter %s is not part of this build (BM3D only)\n", argv[1]);
    return 1;
}
