/* Host side of the NNF download: a small pool of worker threads that turns the packed field the
   GPU sends back (int32 packed position + float32 distance, 8 bytes per patch) into the
   reference's float64 layout ann(y, x, NNF_X | NNF_Y | NNF_DIST) (patchtable.h:175-177, 3500)
   in the caller's buffer.

   Sending the packed field and widening it here moves a third of the bytes over PCIe that the
   float64 field would (8 instead of 24 per patch); the conversion is exact (positions are
   integers below 2^16, a float distance is a double exactly).  The widening of one band of rows
   runs while the GPU still computes and sends the following bands. */
#include <emmintrin.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <condition_variable>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "patchtable_b200.h"
#include "pt_internal.h"

namespace {

class Pool {
public:
    explicit Pool(int n) {
        for (int i = 0; i < n; i++) workers_.emplace_back([this] { loop(); });
    }
    ~Pool() {
        {
            std::lock_guard<std::mutex> g(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto &t : workers_) t.join();
    }
    int size() const { return (int) workers_.size(); }
    /* Runs fn(0) .. fn(parts - 1): parts - 1 on the workers, the last on the caller; returns when all
       have finished.  Calls from several host threads take their turns. */
    void run(int parts, const std::function<void(int)> &fn) {
        if (parts <= 1 || workers_.empty()) {
            for (int i = 0; i < parts; i++) fn(i);
            return;
        }
        std::lock_guard<std::mutex> turn(run_mu_);
        {
            std::lock_guard<std::mutex> g(mu_);
            job_ = &fn;
            next_ = 0;
            parts_ = parts - 1;
            done_ = 0;
            gen_++;
        }
        cv_.notify_all();
        fn(parts - 1);
        std::unique_lock<std::mutex> g(mu_);
        done_cv_.wait(g, [&] { return done_ == parts_; });
        job_ = nullptr;
    }

private:
    void loop() {
        unsigned long long seen = 0;
        for (;;) {
            std::unique_lock<std::mutex> g(mu_);
            cv_.wait(g, [&] { return stop_ || (job_ && gen_ != seen && next_ < parts_); });
            if (stop_) return;
            while (job_ && next_ < parts_) {
                const int i = next_++;
                const std::function<void(int)> *job = job_;
                g.unlock();
                (*job)(i);
                g.lock();
                if (++done_ == parts_) done_cv_.notify_all();
            }
            seen = gen_;
        }
    }

    std::vector<std::thread> workers_;
    std::mutex mu_, run_mu_;
    std::condition_variable cv_, done_cv_;
    const std::function<void(int)> *job_ = nullptr;
    int next_ = 0, parts_ = 0, done_ = 0;
    unsigned long long gen_ = 0;
    bool stop_ = false;
};

std::mutex g_pool_mu;
int g_threads = 0;                 /* 0: not chosen yet */
bool g_widen = true;               /* false: the GPU writes float64 records and they are copied */
std::shared_ptr<Pool> g_pool;      /* a lookup holds its own reference while it widens, so a
                                      pt_set_host_threads meanwhile retires the old pool safely */

int default_threads() {
    const unsigned hw = std::thread::hardware_concurrency();
    return (int) std::max(1u, std::min(8u, hw ? hw : 1u));
}

std::shared_ptr<Pool> pool() {
    std::lock_guard<std::mutex> g(g_pool_mu);
    if (!g_threads) g_threads = default_threads();
    if (!g_pool) g_pool = std::make_shared<Pool>(g_threads - 1);      /* the caller is the last worker */
    return g_pool;
}

}  // namespace

bool pt_host_widen() {
    std::lock_guard<std::mutex> g(g_pool_mu);
    return g_widen;
}

/* Records [i0, i1) of the packed field as float64 triples.  Pairs of patches (48 bytes) go out as
   three 16-byte streaming stores when the destination is 16-byte aligned, so the output lines are
   written without first being read into the cache. */
static void widen_range(const int *pos, const float *dist, long long i0, long long i1, double *ann) {
    long long i = i0;
    auto one = [&](long long k) {
        const int v = pos[k];
        double *o = ann + 3 * k;
        o[0] = pt_x(v);
        o[1] = pt_y(v);
        o[2] = dist[k];
    };
    if (i < i1 && (((uintptr_t) (ann + 3 * i)) & 15)) one(i++);
    for (; i + 2 <= i1; i += 2) {
        const int v0 = pos[i], v1 = pos[i + 1];
        double *o = ann + 3 * i;
        _mm_stream_pd(o, _mm_set_pd((double) pt_y(v0), (double) pt_x(v0)));
        _mm_stream_pd(o + 2, _mm_set_pd((double) pt_x(v1), (double) dist[i]));
        _mm_stream_pd(o + 4, _mm_set_pd((double) dist[i + 1], (double) pt_y(v1)));
    }
    if (i < i1) one(i);
    _mm_sfence();
}

void pt_expand_nnf(const int *pos, const float *dist, long long n, double *ann) {
    if (n <= 0) return;
    const std::shared_ptr<Pool> keep = pool();
    Pool &pl = *keep;
    const int parts = (int) std::min<long long>(pl.size() + 1, std::max<long long>(1, n / 4096));
    long long per = (n + parts - 1) / parts;
    per = (per + 1) & ~1ll;                 /* even: a part's pairs keep the alignment of the whole */
    pl.run(parts, [&](int k) {
        const long long i0 = std::min(n, k * per), i1 = std::min(n, i0 + per);
        widen_range(pos, dist, i0, i1, ann);
    });
}

void pt_host_copy(float *dst, const float *src, size_t n) {
    if (n == 0) return;
    const std::shared_ptr<Pool> keep = pool();
    Pool &pl = *keep;
    const int parts = (int) std::min<size_t>((size_t) pl.size() + 1, std::max<size_t>(1, n / 65536));
    const size_t per = (n + parts - 1) / parts;
    pl.run(parts, [&](int k) {
        const size_t i0 = std::min(n, (size_t) k * per), i1 = std::min(n, i0 + per);
        if (i1 > i0) memcpy(dst + i0, src + i0, sizeof(float) * (i1 - i0));
    });
}

extern "C" int pt_set_host_threads(int n) {
    std::lock_guard<std::mutex> g(g_pool_mu);
    const int old = !g_widen ? -1 : (g_threads ? g_threads : default_threads());
    g_widen = n >= 0;
    const int want = n > 0 ? std::min(n, 256) : default_threads();
    if (want != g_threads) {
        g_pool.reset();         /* the old workers are joined once no lookup holds the pool */
        g_threads = want;
    }
    return old;
}
