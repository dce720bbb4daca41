/*
 * Oracle harness around the reference's own anatomy mapping.
 *
 * Test infrastructure only: compiled together with the reference's
 * unmodified Glioma/Glioma_ReactionDiffusion.cpp and MRAG sources (see
 * oracle/Makefile) into oracle/_ref/ic_harness_{f64,f32}.  It builds the
 * uniform MRAG Grid the reference constructs before its first refinement
 * (Glioma_ReactionDiffusion.cpp:30-35) and calls the reference's
 * Glioma_ReactionDiffusion::_ic (:79-172), which reads {prefix}GM.dat,
 * {prefix}WM.dat and {prefix}CSF.dat, on it.  _ic is a private static member,
 * so this file alone sees the class with its members public; the layout and
 * the compiled function are the reference's.
 *
 *   ic_harness <prefix> <bpd> <icx> <icy> <icz> <out>
 *       out: float64 L, then p_w, p_g, p_csf, phi as n^3 float64 each
 *       (n = 8 * bpd, x fastest); prints one JSON line with the seconds
 *       _ic took (file reads included).
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <vector>
#include <map>
#include <set>
#include <string>
#include <algorithm>
#include <iostream>
#include <fstream>
#include <sys/time.h>

#define private public
#include "Glioma_ReactionDiffusion.h"
#undef private

static int harnessStencil[2][3] = {
    {-1, -1, -1},
    {+2, +2, +2}
};

static double wall_seconds()
{
    struct timeval tv;
    gettimeofday(&tv, NULL);
    return tv.tv_sec + 1e-6 * tv.tv_usec;
}

int main(int argc, char **argv)
{
    if (argc != 7) {
        fprintf(stderr, "usage: %s <prefix> <bpd> <icx> <icy> <icz> <out>\n", argv[0]);
        return 2;
    }
    const std::string prefix = argv[1];
    const int bpd = atoi(argv[2]);
    Real ic[3] = {(Real)atof(argv[3]), (Real)atof(argv[4]), (Real)atof(argv[5])};
    const int n = 8 * bpd;

    Grid<W, B> grid(bpd, bpd, bpd, harnessStencil);
    Real L = 0;
    const double t0 = wall_seconds();
    Glioma_ReactionDiffusion::_ic(grid, prefix, L, ic);
    const double t1 = wall_seconds();

    const size_t n3 = (size_t)n * n * n;
    std::vector<double> out(4 * n3, 0.0);
    std::vector<BlockInfo> vInfo = grid.getBlocksInfo();
    for (size_t i = 0; i < vInfo.size(); i++) {
        const BlockInfo &info = vInfo[i];
        B &block = grid.getBlockCollection()[info.blockID];
        for (int iz = 0; iz < B::sizeZ; iz++)
            for (int iy = 0; iy < B::sizeY; iy++)
                for (int ix = 0; ix < B::sizeX; ix++) {
                    const size_t gx = info.index[0] * B::sizeX + ix;
                    const size_t gy = info.index[1] * B::sizeY + iy;
                    const size_t gz = info.index[2] * B::sizeZ + iz;
                    const size_t g = gx + n * (gy + n * gz);
                    out[g] = block(ix, iy, iz).p_w;
                    out[n3 + g] = block(ix, iy, iz).p_g;
                    out[2 * n3 + g] = block(ix, iy, iz).p_csf;
                    out[3 * n3 + g] = block(ix, iy, iz).phi;
                }
        grid.getBlockCollection().release(info.blockID);
    }
    FILE *f = fopen(argv[6], "wb");
    if (!f) {
        fprintf(stderr, "cannot write %s\n", argv[6]);
        return 1;
    }
    const double Ld = L;
    fwrite(&Ld, sizeof(double), 1, f);
    fwrite(out.data(), sizeof(double), out.size(), f);
    fclose(f);
    printf("{\"ic_seconds\": %.6f, \"n\": %d, \"L\": %.17g}\n", t1 - t0, n, Ld);
    return 0;
}
