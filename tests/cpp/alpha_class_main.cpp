// The reference caller's call sequence (main.cu:376-395) compiled against
// include/Alpha_Shapes_2D.h and libgalpha.so, unchanged in its use of the
// class: gpudtComputeDT, Alpha_Shapes_2D(pInput, pOutput),
// computeAlphaShapes(), the public members and the master-list iterators.
// Test infrastructure: tests/test_alpha_class.py compiles it on the CPU and,
// on a GPU, runs it and compares what it writes with galphaCompute.
//
//   alpha_class_main POINTS.bin OUT.bin
// POINTS.bin: int32 n, then n (x, y) float64 pairs.  OUT.bin: int32 counts
// (nTris, nSpectrum, nPoints, nEdges, nTriList, nMaster, nSpecPtr, status),
// then the triangles, spectrum, point_list, edge_list, tri_list, master_list
// and spec_pointers as the class holds them.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "Alpha_Shapes_2D.h"

// The class's friend: the reference's viewer reads the private interval
// lists through it (Visualizer.cu); here it writes them to a file.
class Visualizer {
public:
    static void write(Alpha_Shapes_2D &as, PGPUDTOUTPUT dt, FILE *f)
    {
        int n[8] = {dt->nTris, (int)as.spectrum.size(), (int)as.point_list.size(), (int)as.edge_list.size(),
                    (int)as.tri_list.size(), (int)as.master_list.size(), (int)as.spec_pointers.size(),
                    as.status()};
        fwrite(n, sizeof(int), 8, f);
        fwrite(dt->triangles, sizeof(gpudtTriangle), dt->nTris, f);
        fwrite(as.spectrum.data(), sizeof(double), as.spectrum.size(), f);
        fwrite(as.point_list.data(), sizeof(point_interval), as.point_list.size(), f);
        fwrite(as.edge_list.data(), sizeof(edge_interval), as.edge_list.size(), f);
        fwrite(as.tri_list.data(), sizeof(triangle_interval), as.tri_list.size(), f);
        fwrite(as.master_list.data(), sizeof(Alpha), as.master_list.size(), f);
        fwrite(as.spec_pointers.data(), sizeof(int), as.spec_pointers.size(), f);
    }
};

int main(int argc, char **argv)
{
    if (argc < 3) return 2;
    FILE *in = fopen(argv[1], "rb");
    if (!in) return 2;
    int n = 0;
    if (fread(&n, sizeof(int), 1, in) != 1 || n <= 0) return 2;
    std::vector<gpudtVertex> pts(n);
    if (fread(pts.data(), sizeof(gpudtVertex), n, in) != (size_t)n) return 2;
    fclose(in);

    GPUDTPARAMS input;
    PGPUDTPARAMS pInput = &input;
    pInput->nPoints = n;
    pInput->points = pts.data();
    pInput->nConstraints = 0;
    pInput->constraints = NULL;
    pInput->minX = pInput->maxX = pts[0].x;
    pInput->minY = pInput->maxY = pts[0].y;
    for (int i = 1; i < n; i++) {
        if (pts[i].x < pInput->minX) pInput->minX = pts[i].x;
        if (pts[i].x > pInput->maxX) pInput->maxX = pts[i].x;
        if (pts[i].y < pInput->minY) pInput->minY = pts[i].y;
        if (pts[i].y > pInput->maxY) pInput->maxY = pts[i].y;
    }
    pInput->fboSize = 1024;

    // main.cu:387-395
    PGPUDTOUTPUT pOutput = NULL;
    if (pOutput) gpudtReleaseDTOutput(pOutput);
    pOutput = gpudtComputeDT(pInput);
    if (!pOutput) return 3;

    Alpha_Shapes_2D as(pInput, pOutput);
    as.computeAlphaShapes();

    // the public interface the viewer uses (Visualizer.cu:151, 293-333)
    long edges = 0;
    for (MasterList_iterator it = as.Master_begin(); it != as.Master_end(); ++it)
        if ((*it).st == EDGE && (*it).at != nu_max) edges++;
    as.setAlpha(as.spectrum.size() > 1 ? as.spectrum[as.spectrum.size() / 2] : 0.0);
    printf("master entries %d (edge ro/nu_min %ld), alpha %.17g\n", (int)as.master_list.size(), edges,
           (double)as.getAlpha());

    FILE *out = fopen(argv[2], "wb");
    if (!out) return 2;
    Visualizer::write(as, pOutput, out);
    fclose(out);
    gpudtReleaseDTOutput(pOutput);
    return as.status() == GPUDT_OK ? 0 : 4;
}
