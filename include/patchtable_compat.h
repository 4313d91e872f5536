/* patchtable_compat.h -- source-compatible drop-in for the reference's C++ PatchTable API.

   Callers written against the reference (patchtable/patchtable_main.cpp:235-309,
   patchtable/analogy.cpp:866-887, patchtable_apps/...) use

       PatchTableParams *p = new PatchTableParams(argc, argv);   // patchtable.cpp:384-387
       PatchTable<> table(p, b, allowed_patches);                // patchtable.h:4397
       double secs = table.lookup(a, ann, ann_prev);             // patchtable.h:4448
       // ann(y, x, NNF_X | NNF_Y | NNF_DIST), float64             // patchtable.h:175-177

   With this header (instead of patchtable.h) and libpatchtable_b200.so the same code runs the
   B200 path.  Array<T> here is a minimal row-major N-d array with the members those callers use
   (sizes, stride, nelems, data, resize, operator(), width/height/channels); it is not the
   reference's full solver/array.h.  Failures print the library's message and exit(1), like the
   reference's ASSERT2 (solver/util.h:32). */
#ifndef PATCHTABLE_COMPAT_H
#define PATCHTABLE_COMPAT_H

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "patchtable_b200.h"

#define NNF_X 0
#define NNF_Y 1
#define NNF_DIST 2

namespace pt_compat_detail {
inline void check(pt_status s, const char *what) {
    if (s != PT_OK) {
        fprintf(stderr, "%s failed (%d): %s\n", what, (int) s, pt_last_error());
        exit(1);
    }
}
}  // namespace pt_compat_detail

/* Minimal Array<T> (solver/array.h:250-340 subset): row-major, sizes/stride/nelems/data. */
template<class real>
class Array {
  public:
    real *data = nullptr;
    std::vector<int> sizes, stride;
    int nelems = 0;
    bool dealloc = true;

    Array() {}
    Array(int h, int w) { resize(std::vector<int>{h, w}); }
    Array(int h, int w, int c) { resize(std::vector<int>{h, w, c}); }
    Array(const Array &o) { assign(o); }
    Array &operator=(const Array &o) { if (this != &o) assign(o); return *this; }
    ~Array() { if (dealloc) delete[] data; }

    void resize(const std::vector<int> &s) {
        if (s == sizes && data) return;
        if (dealloc) delete[] data;
        sizes = s;
        stride.assign(s.size(), 1);
        nelems = 1;
        for (int i = (int) s.size() - 1; i >= 0; i--) { stride[i] = nelems; nelems *= s[i]; }
        data = new real[nelems];
        dealloc = true;
    }
    void resize(int h, int w) { resize(std::vector<int>{h, w}); }
    void resize(int h, int w, int c) { resize(std::vector<int>{h, w, c}); }
    void assign(const Array &o) {
        resize(o.sizes);
        if (nelems) memcpy(data, o.data, sizeof(real) * nelems);
    }
    void clear() { memset(data, 0, sizeof(real) * nelems); }
    int dimensions() const { return (int) sizes.size(); }
    int height() const { return sizes.size() > 0 ? sizes[0] : 1; }
    int width() const { return sizes.size() > 1 ? sizes[1] : 1; }
    int channels() const { return sizes.size() > 2 ? sizes[2] : 1; }
    real &operator()(int y, int x) { return data[y * stride[0] + x * stride[1]]; }
    const real &operator()(int y, int x) const { return data[y * stride[0] + x * stride[1]]; }
    real &operator()(int y, int x, int c) { return data[y * stride[0] + x * stride[1] + c * stride[2]]; }
    const real &operator()(int y, int x, int c) const { return data[y * stride[0] + x * stride[1] + c * stride[2]]; }
};

/* PatchTableParams (patchtable/patchtable_params.h:23-161) over the C struct pt_params. */
class PatchTableParams : public pt_params {
  public:
    std::vector<int> nslices_v;
    PatchTableParams() { pt_params_default(this); }
    PatchTableParams(int argc, char **argv) { pt_params_default(this); set_from_switches(argc, (const char **) argv); }
    PatchTableParams(int argc, const char **argv) { pt_params_default(this); set_from_switches(argc, argv); }
    void set_speed(int i) { pt_compat_detail::check(pt_params_set_speed(this, i), "set_speed"); }
    /* Like the reference, the first token is ignored (it stands in argv[0]). */
    void set_from_switches(std::string s) { pt_compat_detail::check(pt_params_from_switches(this, s.c_str()), "set_from_switches"); }
    void set_from_switches(int argc, const char **argv) {
        std::string s;
        for (int i = 0; i < argc; i++) { s += argv[i]; s += ' '; }
        set_from_switches(s);
    }
    void set_from_switches(int argc, char **argv) { set_from_switches(argc, (const char **) argv); }
};

/* PatchTable<real, in_type, itype> (patchtable/patchtable.h:4359-4491). */
template<class real = float, class in_type = float, class itype = int32_t>
class PatchTable {
  public:
    pt_table *t = nullptr;
    PatchTableParams *p;

    PatchTable(PatchTableParams *p_, const Array<in_type> &b, Array<itype> *allowed_patches = NULL) : p(p_) {
        static_assert(sizeof(in_type) == sizeof(float), "the GPU path takes float images");
        pt_compat_detail::check(pt_table_create(p, (const float *) b.data, b.height(), b.width(), b.channels(),
                                                allowed_patches ? (const int32_t *) allowed_patches->data : NULL, &t),
                                "PatchTable");
    }
    ~PatchTable() { pt_table_free(t); }
    PatchTable(const PatchTable &) = delete;
    PatchTable &operator=(const PatchTable &) = delete;

    double lookup(const Array<in_type> &a, Array<double> &ann, Array<double> *ann_prev = NULL,
                  Array<float> *coherence_temporal_sv = NULL) {
        ann.resize(a.height() - 7, a.width() - 7, 3);
        double secs = 0;
        pt_compat_detail::check(pt_table_set_params(t, p), "lookup");
        pt_compat_detail::check(pt_table_lookup(t, (const float *) a.data, a.height(), a.width(), ann.data,
                                                ann_prev ? ann_prev->data : NULL,
                                                coherence_temporal_sv ? coherence_temporal_sv->data : NULL, &secs),
                                "lookup");
        return secs;
    }

    void save(std::string filename) { pt_compat_detail::check(pt_table_save(t, filename.c_str()), "save"); }
};

#endif /* PATCHTABLE_COMPAT_H */
