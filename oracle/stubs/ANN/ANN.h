/* Stand-in declarations for the ANN library names the reference mentions
   (patchtable.h:98, 777-816, 866-1109, 2661-2755).  ANN is only reached through non-default
   options (-kcoherence_algo ann, -ann 1, -lookup_algo treecann); every entry point aborts. */
#ifndef PTSTUB_ANN_H
#define PTSTUB_ANN_H
#include <cstdio>
#include <cstdlib>
typedef double ANNcoord;
typedef double ANNdist;
typedef int ANNidx;
typedef ANNcoord *ANNpoint;
typedef ANNpoint *ANNpointArray;
inline void ptstub_ann_abort() { fprintf(stderr, "ANN is not available in the oracle build\n"); abort(); }
inline ANNpointArray annAllocPts(int, int) { ptstub_ann_abort(); return 0; }
inline void annDeallocPts(ANNpointArray &) { ptstub_ann_abort(); }
class ANNkd_tree { public:
    ANNkd_tree(ANNpointArray, int, int) { ptstub_ann_abort(); }
    void annkSearch(ANNpoint, int, ANNidx *, ANNdist *, double = 0.0) { ptstub_ann_abort(); }
};
#endif
