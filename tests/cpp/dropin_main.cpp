// Reference-style caller of the C++ drop-in (include/bm3d_b200/BM3D.hpp):
// the BM3D usage of the reference's own harness (source/BM3D.cpp call
// sequence through FilterIF2::process) written exactly as against
// include/BM3D.h. Reads a raw float32 plane, writes basic and final estimates.
//   dropin_main <in.f32> <width> <height> <sigma> <basic_out.f32> <final_out.f32>
#include "bm3d_b200/BM3D.hpp"

#include <cstdio>
#include <cstdlib>

int main(int argc, char **argv)
{
    if (argc != 7) return 2;
    const int w = std::atoi(argv[2]), h = std::atoi(argv[3]);
    const double s = std::atof(argv[4]);
    Plane_FL src(0.f, w, h);
    FILE *f = std::fopen(argv[1], "rb");
    if (!f || std::fread(src.data(), sizeof(float), src.size(), f) != src.size()) return 3;
    std::fclose(f);

    BM3D_Para para("fast");
    para.basic.sigma = {s, s, s};
    para.final.sigma = para.basic.sigma;
    para.thMSE_Default();

    Plane_FL tmp(src, false), dst(src, false);
    BM3D_Basic(para.basic).process(tmp, src, src);
    BM3D_Final(para.final).process(dst, src, tmp);

    Plane_FL both = BM3D(para)(src);  // combined form
    double d = 0;
    for (size_t i = 0; i < both.size(); ++i) {
        double e = both[i] - dst[i];
        d = e * e > d ? e * e : d;
    }
    if (d > 1e-12) return 4;

    FILE *o1 = std::fopen(argv[5], "wb"), *o2 = std::fopen(argv[6], "wb");
    if (!o1 || !o2) return 5;
    std::fwrite(tmp.data(), sizeof(float), tmp.size(), o1);
    std::fwrite(dst.data(), sizeof(float), dst.size(), o2);
    std::fclose(o1);
    std::fclose(o2);
    return 0;
}
