/* Stand-in for the png++ names in solver/array.h:22, 1652-1680, 1777-1815.  The oracle reads and
   writes PFM only (solver/array.h:1646-1660); PNG files abort. */
#ifndef PTSTUB_PNGPP_HPP
#define PTSTUB_PNGPP_HPP
#include <vector>
#include <cstdio>
#include <cstdlib>
namespace png {
struct rgb_pixel { unsigned char red, green, blue;
    rgb_pixel(unsigned char r = 0, unsigned char g = 0, unsigned char b = 0) : red(r), green(g), blue(b) {} };
template<class P> class image { public:
    int w, h; std::vector<P> px;
    image() : w(0), h(0) {}
    image(const char *) : w(0), h(0) { fprintf(stderr, "PNG input is not available in the oracle build; use .pfm\n"); abort(); }
    image(int w_, int h_) : w(w_), h(h_), px((size_t) w_ * h_) {}
    int get_width() const { return w; }
    int get_height() const { return h; }
    P get_pixel(int x, int y) const { return px[(size_t) y * w + x]; }
    P *operator[](int y) { return &px[(size_t) y * w]; }
    void write(const char *) { fprintf(stderr, "PNG output is not available in the oracle build; use .pfm\n"); abort(); }
};
}
#endif
