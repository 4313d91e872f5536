/* Stand-in for the OpenCV names the reference mentions (solver/array.h:37, 95-129, 1441-1545,
   3221-3285; patchtable/patch_pca.h:5-113).  OpenCV is only reached by non-default options
   (-dim_algo pca, image resizing in apps).  The container type works; cv::PCA is the published
   method restated in oracle/pca_jacobi.h (single-channel float data as rows, the mean given or
   sampled), so the reference's own patch sampling and projection loop run; the other
   algorithms abort. */
#ifndef PTSTUB_OPENCV_CORE_HPP
#define PTSTUB_OPENCV_CORE_HPP
#include <vector>
#include <cstdio>
#include <cstdlib>
#include <cstdint>
#include "../../../pca_jacobi.h"
#define PTSTUB_CV_MAKETYPE(depth, cn) ((depth) + (((cn) - 1) << 3))
#define CV_8U 0
#define CV_16U 2
#define CV_32F 5
#define CV_64F 6
#define CV_8UC1 PTSTUB_CV_MAKETYPE(CV_8U, 1)
#define CV_8UC2 PTSTUB_CV_MAKETYPE(CV_8U, 2)
#define CV_8UC3 PTSTUB_CV_MAKETYPE(CV_8U, 3)
#define CV_8UC4 PTSTUB_CV_MAKETYPE(CV_8U, 4)
#define CV_16UC1 PTSTUB_CV_MAKETYPE(CV_16U, 1)
#define CV_16UC2 PTSTUB_CV_MAKETYPE(CV_16U, 2)
#define CV_16UC3 PTSTUB_CV_MAKETYPE(CV_16U, 3)
#define CV_16UC4 PTSTUB_CV_MAKETYPE(CV_16U, 4)
#define CV_32FC1 PTSTUB_CV_MAKETYPE(CV_32F, 1)
#define CV_32FC2 PTSTUB_CV_MAKETYPE(CV_32F, 2)
#define CV_32FC3 PTSTUB_CV_MAKETYPE(CV_32F, 3)
#define CV_32FC4 PTSTUB_CV_MAKETYPE(CV_32F, 4)
#define CV_64FC1 PTSTUB_CV_MAKETYPE(CV_64F, 1)
#define CV_64FC2 PTSTUB_CV_MAKETYPE(CV_64F, 2)
#define CV_64FC3 PTSTUB_CV_MAKETYPE(CV_64F, 3)
#define CV_64FC4 PTSTUB_CV_MAKETYPE(CV_64F, 4)
#define CV_PCA_DATA_AS_ROW 0
namespace cv {
inline void ptstub_cv_abort(const char *what) { fprintf(stderr, "OpenCV %s is not available in the oracle build\n", what); abort(); }
enum { INTER_LANCZOS4 = 4, BORDER_REPLICATE = 1, KMEANS_PP_CENTERS = 2 };
struct Scalar { double v; static Scalar all(double x) { Scalar s; s.v = x; return s; } };
struct Size { int width, height; Size(int w = 0, int h = 0) : width(w), height(h) {} };
struct TermCriteria { enum { COUNT = 1, MAX_ITER = 1, EPS = 2 }; TermCriteria(int = 0, int = 0, double = 0) {} };
class Mat { public:
    int rows, cols, type_;
    std::vector<unsigned char> buf;
    Mat() : rows(0), cols(0), type_(0) {}
    Mat(int r, int c, int t) { create(r, c, t); }
    Mat(int ndims, const int *sizes, int t, const Scalar &) { create(ndims > 0 ? sizes[0] : 0, ndims > 1 ? sizes[1] : 1, t); }
    void create(int r, int c, int t) { rows = r; cols = c; type_ = t; buf.assign((size_t) r * c * elemSize(), 0); }
    int channels() const { return ((type_ >> 3) & 511) + 1; }
    size_t elemSize() const { int d = type_ & 7; size_t s = (d == CV_64F) ? 8 : (d == CV_32F) ? 4 : (d == CV_16U) ? 2 : 1; return s * channels(); }
    template<class T> T *ptr(int r) { return (T *) (buf.data() + (size_t) r * cols * elemSize()); }
    template<class T> const T *ptr(int r) const { return (const T *) (buf.data() + (size_t) r * cols * elemSize()); }
    template<class T> T &at(int i) { return ((T *) buf.data())[i]; }
    static Mat zeros(int r, int c, int t) { return Mat(r, c, t); }
};
class PCA { public:
    std::vector<float> mean_, basis_;
    int d_ = 0, k_ = 0;
    /* data: n x d CV_32FC1 rows; mean: empty (sample mean) or 1 x d CV_32FC1. */
    PCA(const Mat &data, const Mat &mean, int flags, int maxComponents) {
        if (flags != CV_PCA_DATA_AS_ROW || data.type_ != CV_32FC1 || data.rows < 1 ||
            (mean.rows && (mean.rows != 1 || mean.cols != data.cols || mean.type_ != CV_32FC1)))
            ptstub_cv_abort("PCA with these arguments");
        d_ = data.cols;
        k_ = maxComponents > 0 && maxComponents < d_ ? maxComponents : d_;
        pt_pca_jacobi_fit(data.ptr<float>(0), data.rows, d_, mean.rows > 0, mean.rows ? mean.ptr<float>(0) : nullptr, k_,
                          mean_, basis_);
    }
    void project(const Mat &vec, Mat &result) const {
        if (vec.rows != 1 || vec.cols != d_ || vec.type_ != CV_32FC1 || result.rows != 1 || result.cols < k_ ||
            result.type_ != CV_32FC1)
            ptstub_cv_abort("PCA::project with these arguments");
        pt_pca_project(vec.ptr<float>(0), d_, mean_.data(), basis_.data(), k_, result.ptr<float>(0));
    }
};
inline void resize(const Mat &, Mat &, Size, double = 0, double = 0, int = 0) { ptstub_cv_abort("resize"); }
inline void GaussianBlur(const Mat &, Mat &, Size, double, double = 0, int = 0) { ptstub_cv_abort("GaussianBlur"); }
}
#endif
