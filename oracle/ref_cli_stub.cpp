/* The reference CLI (patchtable/patchtable_main.cpp) links the image-analogy app
   (patchtable/analogy.cpp), which needs OpenCV optical flow.  Analogy is outside the
   build/query path, so the oracle CLI links these two stand-ins instead. */
#include <cstdio>
#include <cstdlib>
void analogy(int, char **) { fprintf(stderr, "analogy is not part of the oracle build\n"); exit(1); }
void print_analogy_switches() {}
