/* Exact k-nearest-neighbour search over float points (CPU, test infrastructure).

   The reference's k-coherence step (patchtable/patchtable.h:2653-2987) calls FLANN's
   KDTreeSingleIndex (patchtable.h:822-861, 2415-2432) with checks=1 and eps=5e5, i.e. an
   approximate search whose result depends on FLANN's internal tree layout.  FLANN is not
   vendored in the reference and no version is pinned (README "Install Dependencies"), so the
   oracle replaces it by an EXACT search with a fully specified ranking:

     dist(q, p) = float sum over dims in index order of (q[i]-p[i])*(q[i]-p[i]),
                  each product and each addition rounded to float (no fused multiply-add);
     order      = ascending (dist, point index).

   The CUDA k-coherence kernels implement the same ranking, so the k-coherence sets are
   comparable bit for bit.  The tree below is an ordinary kd-tree (median split on the widest
   dimension, leaves of at most 16 points) with a lower-bound test that keeps every point whose
   distance could tie the current k-th best; it only affects speed, never the result. */
#ifndef PT_ORACLE_KNN_EXACT_H
#define PT_ORACLE_KNN_EXACT_H

#include <vector>
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <cmath>

namespace ptoracle {

/* Squared distance with the ranking's rounding order.  `volatile` keeps the compiler from
   contracting the multiply and the add into one fused operation on targets that have one. */
static inline float knn_dist(const float *a, const float *b, int d) {
    float s = 0.0f;
    for (int i = 0; i < d; i++) {
        volatile float t = a[i] - b[i];
        volatile float t2 = t * t;
        s = s + t2;
    }
    return s;
}

struct KnnResult {
    float dist;
    int idx;
};

static inline bool knn_less(const KnnResult &a, const KnnResult &b) {
    return a.dist < b.dist || (a.dist == b.dist && a.idx < b.idx);
}

class ExactKnn {
  public:
    int n = 0, d = 0;
    std::vector<float> pts;      /* n x d, row-major, in caller's index order */
    std::vector<int> order;      /* permutation: leaves store contiguous ranges of this */
    struct Node { int lo, hi, dim, left, right; float split; };
    std::vector<Node> nodes;

    ExactKnn() {}
    ExactKnn(const float *data, int n_, int d_) { build(data, n_, d_); }

    void build(const float *data, int n_, int d_) {
        n = n_; d = d_;
        pts.assign(data, data + (size_t) n * d);
        order.resize(n);
        for (int i = 0; i < n; i++) order[i] = i;
        nodes.clear();
        nodes.reserve(2 * (n / 8 + 1));
        if (n > 0) build_node(0, n);
    }

    /* Returns the k nearest points of q (k <= n), ascending by (dist, idx). */
    void query(const float *q, int k, std::vector<KnnResult> &out) const {
        out.clear();
        if (n == 0 || k <= 0) return;
        if (k > n) k = n;
        std::vector<KnnResult> best;
        best.reserve(k + 1);
        std::vector<double> off(d, 0.0);
        search(0, q, k, best, 0.0, off);
        out = best;
    }

  private:
    int build_node(int lo, int hi) {
        int id = (int) nodes.size();
        nodes.push_back(Node{lo, hi, -1, -1, -1, 0.0f});
        if (hi - lo <= 16) return id;
        int best_dim = 0;
        float best_spread = -1.0f;
        for (int j = 0; j < d; j++) {
            float mn = pts[(size_t) order[lo] * d + j], mx = mn;
            for (int i = lo + 1; i < hi; i++) {
                float v = pts[(size_t) order[i] * d + j];
                mn = std::min(mn, v); mx = std::max(mx, v);
            }
            if (mx - mn > best_spread) { best_spread = mx - mn; best_dim = j; }
        }
        int mid = (lo + hi) / 2;
        const float *P = pts.data();
        int dd = d, dim = best_dim;
        std::nth_element(order.begin() + lo, order.begin() + mid, order.begin() + hi,
                         [P, dd, dim](int a, int b) {
                             float va = P[(size_t) a * dd + dim], vb = P[(size_t) b * dd + dim];
                             return va < vb || (va == vb && a < b);
                         });
        float split = P[(size_t) order[mid] * d + dim];
        int l = build_node(lo, mid);
        int r = build_node(mid, hi);
        nodes[id].dim = dim;
        nodes[id].split = split;
        nodes[id].left = l;
        nodes[id].right = r;
        return id;
    }

    void consider(const float *q, int k, std::vector<KnnResult> &best, int idx) const {
        KnnResult c{knn_dist(q, &pts[(size_t) idx * d], d), idx};
        if ((int) best.size() == k && !knn_less(c, best.back())) return;
        auto it = std::upper_bound(best.begin(), best.end(), c, knn_less);
        best.insert(it, c);
        if ((int) best.size() > k) best.pop_back();
    }

    void search(int id, const float *q, int k, std::vector<KnnResult> &best, double rd,
                std::vector<double> &off) const {
        const Node &nd = nodes[id];
        if (nd.dim < 0) {
            for (int i = nd.lo; i < nd.hi; i++) consider(q, k, best, order[i]);
            return;
        }
        double diff = (double) q[nd.dim] - (double) nd.split;
        int first = diff < 0 ? nd.left : nd.right;
        int second = diff < 0 ? nd.right : nd.left;
        search(first, q, k, best, rd, off);
        double old = off[nd.dim];
        double rd2 = rd - old * old + diff * diff;
        /* Visit unless every point of the far side is strictly farther than the k-th best;
           the slack absorbs float rounding of the ranked distances. */
        if ((int) best.size() < k || rd2 * (1.0 - 1e-5) <= (double) best.back().dist) {
            off[nd.dim] = diff;
            search(second, q, k, best, rd2, off);
            off[nd.dim] = old;
        }
    }
};

}  /* namespace ptoracle */

#endif
