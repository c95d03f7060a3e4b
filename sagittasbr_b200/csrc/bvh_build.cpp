// bvh_build.cpp -- binned SAH builder (see bvh_build.hpp).
#include "bvh_build.hpp"

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <future>
#include <mutex>
#include <thread>

namespace sbr {
namespace {

struct Box {
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
    float hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    void grow(const float* l, const float* h) {
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], l[a]);
            hi[a] = std::max(hi[a], h[a]);
        }
    }
    void grow(const Box& b) { grow(b.lo, b.hi); }
    double area() const {
        double d[3];
        for (int a = 0; a < 3; ++a) d[a] = std::max(0.0, double(hi[a]) - double(lo[a]));
        return 2.0 * (d[0] * d[1] + d[1] * d[2] + d[2] * d[0]);
    }
};

// Temporary tree node with heap-independent child links (indices into a shared
// pool guarded by a mutex only at allocation).
struct TmpNode {
    Box box;
    int32_t child[2] = {-1, -1};
    int32_t first = 0, count = 0;
};

class Builder {
public:
    Builder(const std::vector<float>& lo, const std::vector<float>& hi, const BuildOptions& opt)
        : lo_(lo), hi_(hi), opt_(opt) {
        n_ = lo.size() / 3;
        idx_.resize(n_);
        cen_.resize(3 * n_);
        for (size_t i = 0; i < n_; ++i) {
            idx_[i] = (int32_t)i;
            for (int a = 0; a < 3; ++a) cen_[3 * i + a] = 0.5f * (lo[3 * i + a] + hi[3 * i + a]);
        }
        int hw = (int)std::thread::hardware_concurrency();
        threads_ = opt.n_threads > 0 ? opt.n_threads : std::max(1, hw);
        pool_.reserve(2 * n_);
    }

    BinTree run() {
        BinTree t;
        if (n_ == 0) return t;
        int root = alloc();
        build(root, 0, (int32_t)n_, 0);
        // renumber in pre-order
        t.nodes.reserve(pool_.size());
        flatten(root, t, 0);
        t.order = idx_;
        return t;
    }

private:
    const std::vector<float>& lo_;
    const std::vector<float>& hi_;
    BuildOptions opt_;
    size_t n_ = 0;
    std::vector<int32_t> idx_;
    std::vector<float> cen_;
    std::vector<TmpNode> pool_;
    std::mutex mu_;
    int threads_ = 1;
    std::atomic<int> live_tasks_{0};

    int alloc() {
        std::lock_guard<std::mutex> g(mu_);
        pool_.emplace_back();
        return (int)pool_.size() - 1;
    }
    TmpNode node_copy(int i) {
        std::lock_guard<std::mutex> g(mu_);
        return pool_[i];
    }
    void node_store(int i, const TmpNode& n) {
        std::lock_guard<std::mutex> g(mu_);
        pool_[i] = n;
    }

    void build(int self, int32_t s, int32_t e, int depth) {
        TmpNode nd;
        Box cb;
        for (int32_t i = s; i < e; ++i) {
            int32_t t = idx_[i];
            nd.box.grow(&lo_[3 * t], &hi_[3 * t]);
            cb.grow(&cen_[3 * t], &cen_[3 * t]);
        }
        nd.first = s;
        nd.count = e - s;
        int32_t n = e - s;
        int32_t mid = -1;
        if (n > opt_.leaf_size) mid = split(s, e, nd.box, cb);
        if (mid < 0) {
            node_store(self, nd);
            return;
        }
        int l = alloc(), r = alloc();
        nd.child[0] = l;
        nd.child[1] = r;
        node_store(self, nd);
        bool par = n >= 16384 && live_tasks_.load() < threads_ - 1;
        if (par) {
            live_tasks_++;
            auto fut = std::async(std::launch::async, [&, l, s, mid, depth] { build(l, s, mid, depth + 1); });
            build(r, mid, e, depth + 1);
            fut.get();
            live_tasks_--;
        } else {
            build(l, s, mid, depth + 1);
            build(r, mid, e, depth + 1);
        }
    }

    // Returns the split position, or -1 to make a leaf.
    int32_t split(int32_t s, int32_t e, const Box& box, const Box& cb) {
        const int B = std::max(2, opt_.bin_count);
        const int32_t n = e - s;
        double parent = box.area();
        double bestCost = INFINITY;
        int bestAx = -1, bestBin = -1;
        std::vector<Box> bins(B), right(B);
        std::vector<int32_t> cnt(B), rcnt(B);
        for (int ax = 0; ax < 3; ++ax) {
            float c0 = cb.lo[ax], ext = cb.hi[ax] - cb.lo[ax];
            if (!(ext > 0.0f)) continue;
            float scl = float(B) / ext;
            std::fill(bins.begin(), bins.end(), Box());
            std::fill(cnt.begin(), cnt.end(), 0);
            for (int32_t i = s; i < e; ++i) {
                int32_t t = idx_[i];
                int b = std::min(B - 1, std::max(0, int((cen_[3 * t + ax] - c0) * scl)));
                bins[b].grow(&lo_[3 * t], &hi_[3 * t]);
                cnt[b]++;
            }
            Box acc;
            int32_t ac = 0;
            for (int b = B - 1; b > 0; --b) {
                acc.grow(bins[b]);
                ac += cnt[b];
                right[b] = acc;
                rcnt[b] = ac;
            }
            acc = Box();
            ac = 0;
            for (int b = 0; b < B - 1; ++b) {
                acc.grow(bins[b]);
                ac += cnt[b];
                if (ac == 0 || rcnt[b + 1] == 0) continue;
                double cost = (acc.area() * ac + right[b + 1].area() * rcnt[b + 1]) / std::max(parent, 1e-300);
                if (cost < bestCost) {
                    bestCost = cost;
                    bestAx = ax;
                    bestBin = b;
                }
            }
        }
        // leaf when the SAH finds no split worth its traversal step and the leaf fits
        if (bestAx >= 0 && (bestCost < double(n) || n > opt_.max_leaf)) {
            float c0 = cb.lo[bestAx], ext = cb.hi[bestAx] - cb.lo[bestAx];
            float scl = float(B) / ext;
            auto it = std::partition(idx_.begin() + s, idx_.begin() + e, [&](int32_t t) {
                int b = std::min(B - 1, std::max(0, int((cen_[3 * t + bestAx] - c0) * scl)));
                return b <= bestBin;
            });
            int32_t mid = int32_t(it - idx_.begin());
            if (mid > s && mid < e) return mid;
        }
        if (n <= opt_.max_leaf) return -1;
        // median split on the widest centroid axis (degenerate centroids included)
        int ax = 0;
        float best = -1.0f;
        for (int a = 0; a < 3; ++a) {
            float ext = cb.hi[a] - cb.lo[a];
            if (ext > best) { best = ext; ax = a; }
        }
        int32_t mid = s + n / 2;
        std::nth_element(idx_.begin() + s, idx_.begin() + mid, idx_.begin() + e, [&](int32_t x, int32_t y) {
            float cx = cen_[3 * x + ax], cy = cen_[3 * y + ax];
            return cx < cy || (cx == cy && x < y);
        });
        return mid;
    }

    int flatten(int src, BinTree& t, int depth) {
        t.depth = std::max(t.depth, depth + 1);
        const TmpNode& n = pool_[src];
        int me = (int)t.nodes.size();
        BinNode b;
        for (int a = 0; a < 3; ++a) { b.lo[a] = n.box.lo[a]; b.hi[a] = n.box.hi[a]; }
        b.left = b.right = -1;
        b.first = n.first;
        b.count = n.count;
        t.nodes.push_back(b);
        if (n.child[0] >= 0) {
            int l = flatten(n.child[0], t, depth + 1);
            int r = flatten(n.child[1], t, depth + 1);
            t.nodes[me].left = l;
            t.nodes[me].right = r;
            t.nodes[me].first = 0;
            t.nodes[me].count = 0;
        }
        return me;
    }
};

}  // namespace

BinTree build_sah(const std::vector<float>& tri_lo, const std::vector<float>& tri_hi, const BuildOptions& opt) {
    Builder b(tri_lo, tri_hi, opt);
    return b.run();
}

}  // namespace sbr
