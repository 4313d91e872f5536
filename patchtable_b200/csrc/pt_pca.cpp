/* -dim_algo pca: the patch basis of the table image (get_patch_pca, patchtable/patch_pca.h:45-52).

   The reference samples pca_samples patches at (rand() % (w-7), rand() % (h-7)) of the colour-
   converted image (extract_patches, patch_pca.h:14-43), each a 192-vector whose entry (row dy,
   column dx, channel c) is float dx + c of the interleaved patch row (the row pointer is indexed
   by dx floats, patch_pca.h:31-36, not by pixels), and hands them to cv::PCA with DATA_AS_ROW and maxComponents = ndims: the sample mean
   (or zero when pca_subtract_mean is off) and the leading eigenvectors of the covariance
   (1/n) sum (x - mean)(x - mean)^T.  OpenCV is not part of this build, so the decomposition is
   the published cyclic Jacobi method, in double precision; eigenvectors are ordered by
   decreasing eigenvalue and signed so that their largest-magnitude entry is positive (OpenCV
   leaves the sign to its solver).  The fit runs on the host: a thousand samples and a 192 x 192
   matrix; the projection of every patch runs on the GPU (k_descriptor.cu). */
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <numeric>
#include <memory>
#include <vector>

#include "pt_internal.h"
#include "pt_kernels.h"

namespace {

/* ARRAY_RGB2YUV (solver/array.h:1124-1126) in double, as the GPU descriptor kernels compute it. */
inline void yuv_host(float R, float G, float B, float &Y, float &U, float &V) {
    const double r = R, g = G, b = B;
    Y = (float) ((0.299 * r + 0.587 * g) + 0.114 * b);
    U = (float) ((-0.14713 * r + -0.28886 * g) + 0.436 * b);
    V = (float) ((0.615 * r + -0.51499 * g) + -0.10001 * b);
}

/* Array::rgb2lab as the GPU descriptor kernels compute it (k_descriptor.cu: lab_exact). */
struct LabHost {
    float tab[2][PT_LAB_N];
    LabHost() { pt_lab_pow_tables(tab); }
    float look(int t, float v) const {
        int i = (int) (v * (float) PT_LAB_N);
        i = i < 0 ? 0 : (i >= PT_LAB_N ? PT_LAB_N - 1 : i);
        return tab[t][i];
    }
    float lin(float c) const {
        const double cd = c;
        if (cd <= 0.04045) return (float) (cd / 12.92);
        return look(0, (float) ((cd + 0.055) / 1.055));
    }
    float f(float r) const {
        if ((double) r > 0.008856) return look(1, r);
        return (float) ((903.3 * (double) r + 16.0) / 116.0);
    }
    void operator()(float R, float G, float B, float &L, float &A, float &Bo) const {
        const double r = lin(R), g = lin(G), b = lin(B);
        const float X = (float) ((0.4360747 * r + 0.3850649 * g) + 0.1430804 * b);
        const float Y = (float) ((0.2225045 * r + 0.7168786 * g) + 0.0606169 * b);
        const float Z = (float) ((0.0139322 * r + 0.0971045 * g) + 0.7141733 * b);
        const float fx = f((float) ((double) X / 0.9642)), fy = f((float) ((double) Y / 1.0)),
                    fz = f((float) ((double) Z / 0.8249));
        L = 116.0f * fy - 16.0f;
        A = 500.0f * (fx - fy);
        Bo = 200.0f * (fy - fz);
    }
};

/* Eigen-decomposition of the symmetric n x n matrix a (row-major, destroyed) by cyclic Jacobi
   rotations; vals[k] and column k of vecs (row-major n x n) are the pairs. */
void jacobi_eigen(std::vector<double> &a, int n, std::vector<double> &vals, std::vector<double> &vecs) {
    vecs.assign((size_t) n * n, 0.0);
    for (int i = 0; i < n; i++) vecs[(size_t) i * n + i] = 1.0;
    auto A = [&](int i, int j) -> double & { return a[(size_t) i * n + j]; };
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0.0, diag = 0.0;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) (i == j ? diag : off) += A(i, j) * A(i, j);
        if (off <= 1e-30 * diag || off == 0.0) break;
        for (int p = 0; p < n - 1; p++)
            for (int q = p + 1; q < n; q++) {
                const double apq = A(p, q);
                if (apq == 0.0) continue;
                const double theta = (A(q, q) - A(p, p)) / (2.0 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < n; k++) {           /* columns p, q */
                    const double akp = A(k, p), akq = A(k, q);
                    A(k, p) = c * akp - s * akq;
                    A(k, q) = s * akp + c * akq;
                }
                for (int k = 0; k < n; k++) {           /* rows p, q */
                    const double apk = A(p, k), aqk = A(q, k);
                    A(p, k) = c * apk - s * aqk;
                    A(q, k) = s * apk + c * aqk;
                }
                for (int k = 0; k < n; k++) {
                    double &vkp = vecs[(size_t) k * n + p], &vkq = vecs[(size_t) k * n + q];
                    const double x = vkp, y = vkq;
                    vkp = c * x - s * y;
                    vkq = s * x + c * y;
                }
            }
    }
    vals.resize(n);
    for (int i = 0; i < n; i++) vals[i] = A(i, i);
}

}  // namespace

pt_status pt_pca_fit(const float *rgb, int h, int w, int convert, int samples, int subtract_mean, int ncomp,
                     std::vector<float> &mean_out, std::vector<float> &basis_out) {
    constexpr int D = PT_PCA_DIM;
    if (samples < 1) return pt_fail(PT_BAD_ARG, "pca_samples must be >= 1");
    if (ncomp < 1 || ncomp > PT_DESC_MAX) return pt_fail(PT_UNSUPPORTED, "PCA with %d components", ncomp);
    const int aew = w - 7, aeh = h - 7;
    std::vector<double> X((size_t) samples * D);
    std::unique_ptr<LabHost> lab;
    if (convert == PT_COLOR_LAB) lab.reset(new LabHost());
    for (int i = 0; i < samples; i++) {
        const int ax = rand() % aew;                   /* extract_patches, patch_pca.h:25-26 */
        const int ay = rand() % aeh;
        double *row = &X[(size_t) i * D];
        int k = 0;
        for (int dy = 0; dy < 8; dy++) {
            /* the first four colour-converted pixels of the patch row, interleaved: entry (dy, dx, c)
               is float dx + c of the row (patch_pca.h:31-36 index the row pointer by dx floats) */
            float conv[12];
            for (int q = 0; q < 4; q++) {
                const float *px = rgb + ((size_t) (ay + dy) * w + ax + q) * 3;
                float c0 = px[0], c1 = px[1], c2 = px[2];
                if (convert == PT_COLOR_YUV) yuv_host(px[0], px[1], px[2], c0, c1, c2);
                else if (convert == PT_COLOR_LAB) (*lab)(px[0], px[1], px[2], c0, c1, c2);
                conv[3 * q] = c0; conv[3 * q + 1] = c1; conv[3 * q + 2] = c2;
            }
            for (int dx = 0; dx < 8; dx++)
                for (int c = 0; c < 3; c++) row[k++] = conv[dx + c];
        }
    }
    std::vector<double> mean(D, 0.0);
    if (subtract_mean) {
        for (int i = 0; i < samples; i++)
            for (int j = 0; j < D; j++) mean[j] += X[(size_t) i * D + j];
        for (int j = 0; j < D; j++) mean[j] /= samples;
    }
    std::vector<double> C((size_t) D * D, 0.0);
    for (int i = 0; i < samples; i++) {
        const double *row = &X[(size_t) i * D];
        double d[D];
        for (int j = 0; j < D; j++) d[j] = row[j] - mean[j];
        for (int a = 0; a < D; a++)
            for (int b = a; b < D; b++) C[(size_t) a * D + b] += d[a] * d[b];
    }
    for (int a = 0; a < D; a++)
        for (int b = a; b < D; b++) {
            C[(size_t) a * D + b] /= samples;
            C[(size_t) b * D + a] = C[(size_t) a * D + b];
        }
    std::vector<double> vals, vecs;
    jacobi_eigen(C, D, vals, vecs);
    std::vector<int> order(D);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return vals[x] > vals[y]; });
    mean_out.resize(D);
    for (int j = 0; j < D; j++) mean_out[j] = (float) mean[j];
    basis_out.assign((size_t) ncomp * D, 0.0f);
    for (int k = 0; k < ncomp; k++) {
        const int col = order[k];
        int big = 0;
        for (int j = 1; j < D; j++)
            if (std::fabs(vecs[(size_t) j * D + col]) > std::fabs(vecs[(size_t) big * D + col])) big = j;
        const double sgn = vecs[(size_t) big * D + col] < 0 ? -1.0 : 1.0;
        for (int j = 0; j < D; j++) basis_out[(size_t) k * D + j] = (float) (sgn * vecs[(size_t) j * D + col]);
    }
    return PT_OK;
}

void pt_lab_pow_tables(float (*tab)[PT_LAB_N]) {
    /* PowTable(real p, real upper = 1), solver/array.h:221-237, with p stored as float */
    const float p[2] = {2.4f, (float) (1.0 / 3.0)};
    for (int t = 0; t < 2; t++)
        for (int i = 0; i < PT_LAB_N; i++) {
            const double v = (i + 0.5) / PT_LAB_N * (double) 1.0f;
            tab[t][i] = (float) std::pow(v, (double) p[t]);
        }
}
