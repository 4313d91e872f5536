/* Principal components of sampled patches, shared by the oracle restatement (pt_oracle.cpp) and
   the cv::PCA stand-in that lets the reference's own get_patch_pca / apply_patch_pca
   (patchtable/patch_pca.h:14-113) run in the oracle build (stubs/opencv2/core/core.hpp).
   Test infrastructure only.

   cv::PCA(data, mean, DATA_AS_ROW, maxComponents) is restated from its published definition:
   the mean is the sample mean of the rows, or the given mean (patch_pca.h passes zeros when
   pca_subtract_mean is off); the covariance is (1/n) sum (x - mean)(x - mean)^T; its
   eigenvectors come from the cyclic Jacobi method (rotations over every pair (r, q), r < q, in
   row order, until the off-diagonal mass is below 1e-30 of the diagonal's), ordered by decreasing
   eigenvalue and signed so that the entry of largest magnitude is positive.  Everything is
   computed in double and stored as float, as OpenCV stores a CV_32F model.  OpenCV's own solver
   is not available here, so parity with the original library is not claimed; what this pins is
   the reference's sampling (rand() order) and projection loop around the decomposition. */
#ifndef PT_ORACLE_PCA_JACOBI_H
#define PT_ORACLE_PCA_JACOBI_H

#include <algorithm>
#include <cmath>
#include <vector>

/* X: n rows of d floats.  With use_mean, mean_in (d floats) is the mean; otherwise the sample
   mean.  Writes mean_out (d) and basis (ncomp x d, row k = component k). */
inline void pt_pca_jacobi_fit(const float *X, int n, int d, bool use_mean, const float *mean_in, int ncomp,
                              std::vector<float> &mean_out, std::vector<float> &basis) {
    std::vector<double> mu(d, 0.0);
    if (use_mean) {
        for (int j = 0; j < d; j++) mu[j] = mean_in[j];
    } else {
        for (int i = 0; i < n; i++)
            for (int j = 0; j < d; j++) mu[j] += (double) X[(size_t) i * d + j];
        for (int j = 0; j < d; j++) mu[j] /= n;
    }
    std::vector<double> A((size_t) d * d, 0.0);
    for (int i = 0; i < n; i++)
        for (int a = 0; a < d; a++) {
            const double da = (double) X[(size_t) i * d + a] - mu[a];
            for (int b = a; b < d; b++) A[(size_t) a * d + b] += da * ((double) X[(size_t) i * d + b] - mu[b]);
        }
    for (int a = 0; a < d; a++)
        for (int b = a; b < d; b++) { A[(size_t) a * d + b] /= n; A[(size_t) b * d + a] = A[(size_t) a * d + b]; }
    std::vector<double> V((size_t) d * d, 0.0);
    for (int i = 0; i < d; i++) V[(size_t) i * d + i] = 1.0;
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0.0, on = 0.0;
        for (int i = 0; i < d; i++)
            for (int j = 0; j < d; j++) {
                const double v = A[(size_t) i * d + j];
                if (i == j) on += v * v; else off += v * v;
            }
        if (off == 0.0 || off <= 1e-30 * on) break;
        for (int r = 0; r < d - 1; r++)
            for (int q = r + 1; q < d; q++) {
                const double arq = A[(size_t) r * d + q];
                if (arq == 0.0) continue;
                const double theta = (A[(size_t) q * d + q] - A[(size_t) r * d + r]) / (2.0 * arq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), sn = t * c;
                for (int k = 0; k < d; k++) {
                    const double x = A[(size_t) k * d + r], y = A[(size_t) k * d + q];
                    A[(size_t) k * d + r] = c * x - sn * y;
                    A[(size_t) k * d + q] = sn * x + c * y;
                }
                for (int k = 0; k < d; k++) {
                    const double x = A[(size_t) r * d + k], y = A[(size_t) q * d + k];
                    A[(size_t) r * d + k] = c * x - sn * y;
                    A[(size_t) q * d + k] = sn * x + c * y;
                }
                for (int k = 0; k < d; k++) {
                    const double x = V[(size_t) k * d + r], y = V[(size_t) k * d + q];
                    V[(size_t) k * d + r] = c * x - sn * y;
                    V[(size_t) k * d + q] = sn * x + c * y;
                }
            }
    }
    std::vector<int> ord(d);
    for (int i = 0; i < d; i++) ord[i] = i;
    std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return A[(size_t) x * d + x] > A[(size_t) y * d + y]; });
    mean_out.resize(d);
    for (int j = 0; j < d; j++) mean_out[j] = (float) mu[j];
    basis.assign((size_t) ncomp * d, 0.0f);
    for (int k = 0; k < ncomp && k < d; k++) {
        const int col = ord[k];
        int big = 0;
        for (int j = 1; j < d; j++)
            if (std::fabs(V[(size_t) j * d + col]) > std::fabs(V[(size_t) big * d + col])) big = j;
        const double sg = V[(size_t) big * d + col] < 0 ? -1.0 : 1.0;
        for (int j = 0; j < d; j++) basis[(size_t) k * d + j] = (float) (sg * V[(size_t) j * d + col]);
    }
}

/* cv::PCA::project of one DATA_AS_ROW vector: out[k] = sum_j (v_j - mean_j) * basis_kj, summed in
   j order in float. */
inline void pt_pca_project(const float *v, int d, const float *mean, const float *basis, int ncomp, float *out) {
    for (int k = 0; k < ncomp; k++) {
        float acc = 0.0f;
        for (int j = 0; j < d; j++) acc = acc + (v[j] - mean[j]) * basis[(size_t) k * d + j];
        out[k] = acc;
    }
}

#endif
