// Reference-style caller of the C++ drop-in on integer planes and RGB frames:
// the usage of the reference's BM3D classes on Plane / Frame
// (FilterIF2::operator() and process, include/Filter.h:138-217) written as
// against include/BM3D.h. Reads a raw planar RGB int32 frame, writes
//   the combined filter's frame, the basic stage's frame, the final stage's
//   frame (ref = the basic frame), and the combined filter on the R plane alone.
//   dropin_frame <in.i32> <width> <height> <sigma> <out.i32>
#include "bm3d_b200/BM3D.hpp"

#include <cstdio>
#include <cstdlib>
#include <vector>

int main(int argc, char **argv)
{
    if (argc != 6) return 2;
    const int w = std::atoi(argv[2]), h = std::atoi(argv[3]);
    const double s = std::atof(argv[4]);
    Frame src(0, w, h, 8, true);
    FILE *f = std::fopen(argv[1], "rb");
    if (!f) return 3;
    for (int c = 0; c < 3; ++c)
        if (std::fread(src.P(c).data(), sizeof(int32_t), static_cast<size_t>(w) * h, f) !=
            static_cast<size_t>(w) * h)
            return 3;
    std::fclose(f);

    BM3D_Para para("fast");
    para.basic.sigma = {s, s, s};
    para.final.sigma = para.basic.sigma;
    para.thMSE_Default();

    Frame full = BM3D(para)(src);
    Frame basic = BM3D_Basic(para.basic)(src);
    Frame fin(src, false);
    BM3D_Final(para.final).process(fin, src, basic);
    Plane r_full = BM3D(para)(src.R());

    FILE *o = std::fopen(argv[5], "wb");
    if (!o) return 5;
    for (const Frame *fr : {&full, &basic, &fin})
        for (int c = 0; c < 3; ++c)
            std::fwrite(fr->P(c).data(), sizeof(int32_t), static_cast<size_t>(w) * h, o);
    std::fwrite(r_full.data(), sizeof(int32_t), static_cast<size_t>(w) * h, o);
    std::fclose(o);
    return 0;
}
