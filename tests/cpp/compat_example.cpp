/* A reference-style caller (patchtable/patchtable_main.cpp:235-309) compiled against
   include/patchtable_compat.h: builds a table on b.raw, queries a.raw, prints the mean NNF
   distance (get_mean_dist, patchtable_main.cpp:90-101) and writes the NNF.
   Usage: compat_example h w a.raw b.raw out.raw [switches...]  (raw float32 h x w x 3 images). */
#include <cmath>
#include <cstdio>
#include <cstdlib>

#include "patchtable_compat.h"

static void read_raw(const char *fn, Array<float> &img) {
    FILE *f = fopen(fn, "rb");
    if (!f || fread(img.data, sizeof(float), img.nelems, f) != (size_t) img.nelems) { fprintf(stderr, "read %s\n", fn); exit(1); }
    fclose(f);
}

int main(int argc, char **argv) {
    if (argc < 6) { fprintf(stderr, "usage: compat_example h w a.raw b.raw out.raw [switches]\n"); return 2; }
    int h = atoi(argv[1]), w = atoi(argv[2]);
    Array<float> a(h, w, 3), b(h, w, 3);
    read_raw(argv[3], a);
    read_raw(argv[4], b);
    PatchTableParams *p = new PatchTableParams(argc - 5, argv + 5);   /* argv[5] takes the argv[0] slot */
    PatchTable<> table(p, b);
    Array<double> ann;
    double secs = table.lookup(a, ann);
    double mean = 0;
    for (int y = 0; y < ann.height(); y++)
        for (int x = 0; x < ann.width(); x++) { double d = ann(y, x, NNF_DIST); mean += std::sqrt(d < 0 ? 0 : d); }
    mean /= double(ann.height() * ann.width());
    printf("1-NN overall lookup time: %f secs\nmean_dist: %f\n", secs, mean);
    FILE *f = fopen(argv[5], "wb");
    fwrite(ann.data, sizeof(double), ann.nelems, f);
    fclose(f);
    delete p;
    return 0;
}
