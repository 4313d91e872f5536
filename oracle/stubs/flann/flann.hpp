/* Stand-in for the FLANN interface the reference calls (patchtable.h:81, 819-861, 2214-2230,
   2415-2432, 2653-2760).  FLANN is not vendored and no version is pinned by the reference, so
   this stand-in answers knnSearch EXACTLY with the ranking documented in oracle/knn_exact.h:
   ascending (float squared L2 distance summed in dimension order, point index).  Parity for the
   k-coherence step is therefore pinned to this exact search, not to FLANN's approximate one. */
#ifndef PTSTUB_FLANN_HPP
#define PTSTUB_FLANN_HPP
#include <vector>
#include <cstddef>
#include "../../knn_exact.h"
namespace flann {
template<class T> struct L2 { typedef T ElementType; typedef T ResultType; };
template<class T> class Matrix { public:
    T *data; size_t rows, cols;
    Matrix() : data(0), rows(0), cols(0) {}
    Matrix(T *d, size_t r, size_t c) : data(d), rows(r), cols(c) {}
    T *operator[](size_t i) const { return data + i * cols; }
    T *ptr() const { return data; }
};
struct IndexParams { virtual ~IndexParams() {} };
struct KDTreeSingleIndexParams : IndexParams { KDTreeSingleIndexParams(int = 10, bool = false) {} };
struct KDTreeIndexParams : IndexParams { KDTreeIndexParams(int = 4) {} };
struct LinearIndexParams : IndexParams { LinearIndexParams() {} };
struct SearchParams { int checks; float eps; bool sorted;
    SearchParams(int c = 32, float e = 0.0f, bool s = true) : checks(c), eps(e), sorted(s) {} };
template<class Distance> class Index { public:
    typedef typename Distance::ElementType ElementType;
    ptoracle::ExactKnn knn;
    Index(const Matrix<ElementType> &data, const IndexParams &) {
        knn.build(data.data, (int) data.rows, (int) data.cols);
    }
    void buildIndex() {}
    int knnSearch(const Matrix<ElementType> &queries, std::vector<std::vector<int> > &indices,
                  std::vector<std::vector<float> > &dists, size_t k, const SearchParams &) {
        std::vector<ptoracle::KnnResult> res;
        indices.resize(queries.rows);
        dists.resize(queries.rows);
        for (size_t i = 0; i < queries.rows; i++) {
            knn.query(queries[i], (int) k, res);
            indices[i].assign(k, -1);
            dists[i].assign(k, 0.0f);
            for (size_t j = 0; j < res.size(); j++) { indices[i][j] = res[j].idx; dists[i][j] = res[j].dist; }
        }
        return (int) queries.rows;
    }
};
}
#endif
