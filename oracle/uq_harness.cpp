/*
 * The reference's own UQ dump (Glioma_ReactionDiffusion::_dumpUQoutput,
 * Glioma/Glioma_ReactionDiffusion.cpp:208-262) of an adapted grid: the
 * values the oracle's uq_dump restates.  Test infrastructure: compiled with
 * the reference's unmodified Glioma_ReactionDiffusion.cpp and MRAG sources
 * (oracle/Makefile, target ref); no GPU.  As in ic_harness.cpp, the class's
 * private members are visible to this harness alone.
 *
 *   uq_harness <prefix> <icx> <icy> <icz> <refine_tol> <compress_tol> <outdir> [sigma]
 *
 * Constructs the reference's Glioma_ReactionDiffusion as the brain program
 * does for "-model RD" (its grid of _BPD_^3 blocks and _ic on
 * <prefix>GM.dat, WM.dat, CSF.dat with the tumour at (icx, icy, icz)); with
 * sigma > 0 phi is then replaced by exp(-|x - ic|^2 / (2 sigma^2)), so that
 * coarse blocks carry values too.  It adapts the grid with
 * Science::AutomaticRefinement (up to _MAXLEVEL_) and
 * Science::AutomaticCompression with the given tolerances, writes the leaves
 * to <outdir>/leaves.bin (records: int32 name length, name, int32 kind
 * (0 int64, 1 float64), int64 count, data: level, index (3 per leaf), h (the
 * Real spacing), phi (512 per leaf, x fastest)) and calls _dumpUQoutput in
 * <outdir>, which writes HGG_data.dat.  Prints one JSON line.
 */
#include <unistd.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <set>
#include <string>
#include <vector>

#define private public
#include "Glioma_ReactionDiffusion.h"
#undef private

static void put(FILE *f, const char *name, int kind, const void *data, int64_t n)
{
    const int len = (int)strlen(name);
    fwrite(&len, 4, 1, f);
    fwrite(name, 1, len, f);
    fwrite(&kind, 4, 1, f);
    fwrite(&n, 8, 1, f);
    if (n) fwrite(data, 8, n, f);
}

int main(int argc, char **argv)
{
    if (argc != 8 && argc != 9) {
        fprintf(stderr, "usage: %s <prefix> <icx> <icy> <icz> <refine_tol> <compress_tol> <outdir> [sigma]\n",
                argv[0]);
        return 2;
    }
    const double sigma = argc == 9 ? atof(argv[8]) : 0.0;
    const char *args[] = {"brain", "-PatFileName", argv[1], "-icx", argv[2], "-icy", argv[3], "-icz", argv[4],
                          "-verbose", "0", "-vtk", "0", "-bDumpIC", "0", "-UQ", "0", "-adaptive", "1",
                          "-dumpfreq", "1"};
    const int nargs = (int)(sizeof(args) / sizeof(args[0]));
    /* never deleted: the destructor only prints */
    Glioma_ReactionDiffusion *sim = new Glioma_ReactionDiffusion(nargs, args);
    Grid<W, B> &grid = *sim->grid;
    if (sigma > 0) {
        const double c[3] = {atof(argv[2]), atof(argv[3]), atof(argv[4])};
        std::vector<BlockInfo> v = grid.getBlocksInfo();
        for (size_t i = 0; i < v.size(); i++) {
            B &block = grid.getBlockCollection()[v[i].blockID];
            for (int iz = 0; iz < B::sizeZ; iz++)
                for (int iy = 0; iy < B::sizeY; iy++)
                    for (int ix = 0; ix < B::sizeX; ix++) {
                        double x[3];
                        v[i].pos(x, ix, iy, iz);
                        const double r2 = (x[0] - c[0]) * (x[0] - c[0]) + (x[1] - c[1]) * (x[1] - c[1]) +
                                          (x[2] - c[2]) * (x[2] - c[2]);
                        block(ix, iy, iz).phi = (Real)exp(-r2 / (2 * sigma * sigma));
                    }
        }
    }
    Science::AutomaticRefinement<0, 0>(grid, sim->blockfwt, atof(argv[5]), maxLevel, -1, NULL);
    Science::AutomaticCompression<0, 0>(grid, sim->blockfwt, atof(argv[6]), -1, NULL);

    std::vector<BlockInfo> vInfo = grid.getBlocksInfo();
    const size_t nb = vInfo.size();
    std::vector<int64_t> level(nb), index(3 * nb);
    std::vector<double> h(nb), phi(nb * 512);
    std::map<int, int> levels;
    for (size_t i = 0; i < nb; i++) {
        level[i] = vInfo[i].level;
        levels[vInfo[i].level]++;
        for (int d = 0; d < 3; d++) index[3 * i + d] = vInfo[i].index[d];
        h[i] = (double)vInfo[i].h[0];
        B &block = grid.getBlockCollection()[vInfo[i].blockID];
        for (int iz = 0; iz < B::sizeZ; iz++)
            for (int iy = 0; iy < B::sizeY; iy++)
                for (int ix = 0; ix < B::sizeX; ix++)
                    phi[i * 512 + ix + 8 * (iy + 8 * iz)] = (double)block(ix, iy, iz).phi;
    }
    if (chdir(argv[7]) != 0) {
        fprintf(stderr, "uq_harness: cannot enter %s\n", argv[7]);
        return 2;
    }
    FILE *f = fopen("leaves.bin", "wb");
    if (!f) return 2;
    put(f, "level", 0, &level[0], (int64_t)nb);
    put(f, "index", 0, &index[0], (int64_t)(3 * nb));
    put(f, "h", 1, &h[0], (int64_t)nb);
    put(f, "phi", 1, &phi[0], (int64_t)(nb * 512));
    fclose(f);
    sim->_dumpUQoutput();

    printf("{\"leaves\": %d, \"gpd\": %d, \"real_bytes\": %d, \"levels\": {", (int)nb, blocksPerDimension * blockSize,
           (int)sizeof(Real));
    for (std::map<int, int>::const_iterator it = levels.begin(); it != levels.end(); ++it)
        printf("%s\"%d\": %d", it == levels.begin() ? "" : ", ", it->first, it->second);
    printf("}}\n");
    fflush(stdout);
    _exit(0);
}
