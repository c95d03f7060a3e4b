// tie_order.cpp -- the reference walk's order over triangles, for exact ties.
//
// The tree is the one the reference's FP64 build makes (src/scene/bvhBuilder.cpp:
// 93-312 with Real = double): binned SAH on centroids over all three axes, 16 bins,
// cost (A_L N_L + A_R N_R) / A_P, no split at a cost >= N, std::partition on
// `centroid < split position`, the std::nth_element median split where SAH finds
// none, leaves of up to 4 triangles.  The steps and their arithmetic are kept
// alike on purpose: the order of triangles inside a leaf, which decides ties, is
// whatever std::partition and std::nth_element leave there.  Only the leaf ranges
// and the final triangle order are kept (the walk order needs nothing else);
// subtrees work on disjoint ranges, so building them on separate threads gives the
// same order.
#include "tie_order.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>

namespace sbr {

namespace {

struct D3 {
    double x, y, z;
    double operator[](int a) const { return a == 0 ? x : (a == 1 ? y : z); }
};
D3 dmin(D3 a, D3 b) { return {std::fmin(a.x, b.x), std::fmin(a.y, b.y), std::fmin(a.z, b.z)}; }
D3 dmax(D3 a, D3 b) { return {std::fmax(a.x, b.x), std::fmax(a.y, b.y), std::fmax(a.z, b.z)}; }

constexpr double kBig = 1.7976931348623158e+308;  // the FP64 build's REAL_FLT_MAX
constexpr int kLeaf = 4;
constexpr int kBins = 16;

struct RefTree {
    std::vector<D3> c, lo, hi;     // per caller triangle: centroid and box
    std::vector<int32_t> perm;     // the reference's triangle order
    std::vector<int32_t> leaf_n;   // leaf_n[s] = triangle count of the leaf starting at s, else 0

    // surface area with negative extents clamped (src/scene/bvhBuilder.cpp:46-52)
    static double area(D3 lo, D3 hi) {
        const double dx = std::fmax(0.0, hi.x - lo.x), dy = std::fmax(0.0, hi.y - lo.y),
                     dz = std::fmax(0.0, hi.z - lo.z);
        return 2.0 * (dx * dy + dy * dz + dz * dx);
    }
    void cbounds(int s, int e, D3& clo, D3& chi) const {
        clo = {kBig, kBig, kBig};
        chi = {-kBig, -kBig, -kBig};
        for (int i = s; i < e; ++i) { clo = dmin(clo, c[perm[i]]); chi = dmax(chi, c[perm[i]]); }
    }
    // src/scene/bvhBuilder.cpp:93-113
    bool split_median(int s, int e, int& mid) {
        D3 clo, chi;
        cbounds(s, e, clo, chi);
        const D3 ext{chi.x - clo.x, chi.y - clo.y, chi.z - clo.z};
        const int ax = (ext.x >= ext.y && ext.x >= ext.z) ? 0 : (ext.y >= ext.z ? 1 : 2);
        mid = s + (e - s) / 2;
        const D3* cc = c.data();
        std::nth_element(perm.begin() + s, perm.begin() + mid, perm.begin() + e,
                         [cc, ax](int32_t a, int32_t b) { return cc[a][ax] < cc[b][ax]; });
        return mid > s && mid < e;
    }
    // src/scene/bvhBuilder.cpp:115-240
    bool split_sah(int s, int e, D3 lo0, D3 hi0, int& mid) {
        D3 clo, chi;
        cbounds(s, e, clo, chi);
        const D3 cext{chi.x - clo.x, chi.y - clo.y, chi.z - clo.z};
        const double parent = area(lo0, hi0);
        if (parent <= 0.0) return false;
        int bestAx = -1, bestSplit = -1;
        double bestCost = kBig;
        D3 blo[kBins], bhi[kBins], llo[kBins], lhi[kBins], rlo[kBins], rhi[kBins];
        int bn[kBins], ln[kBins], rn[kBins];
        for (int ax = 0; ax < 3; ++ax) {
            const double ext = cext[ax];
            if (ext <= 1.0e-6) continue;
            for (int b = 0; b < kBins; ++b) {
                blo[b] = {kBig, kBig, kBig};
                bhi[b] = {-kBig, -kBig, -kBig};
                bn[b] = 0;
            }
            for (int i = s; i < e; ++i) {
                const int32_t t = perm[i];
                const double off = (c[t][ax] - clo[ax]) / ext;
                int b = static_cast<int>(off * kBins);
                b = b < 0 ? 0 : (b >= kBins ? kBins - 1 : b);
                blo[b] = dmin(blo[b], lo[t]);
                bhi[b] = dmax(bhi[b], hi[t]);
                bn[b] += 1;
            }
            D3 rl{kBig, kBig, kBig}, rh{-kBig, -kBig, -kBig};
            int cnt = 0;
            for (int b = 0; b < kBins; ++b) {
                if (bn[b] > 0) { rl = dmin(rl, blo[b]); rh = dmax(rh, bhi[b]); cnt += bn[b]; }
                llo[b] = rl; lhi[b] = rh; ln[b] = cnt;
            }
            rl = {kBig, kBig, kBig};
            rh = {-kBig, -kBig, -kBig};
            cnt = 0;
            for (int b = kBins - 1; b >= 0; --b) {
                if (bn[b] > 0) { rl = dmin(rl, blo[b]); rh = dmax(rh, bhi[b]); cnt += bn[b]; }
                rlo[b] = rl; rhi[b] = rh; rn[b] = cnt;
            }
            for (int b = 0; b < kBins - 1; ++b) {
                const int nl = ln[b], nr = rn[b + 1];
                if (nl == 0 || nr == 0) continue;
                const double cost = (area(llo[b], lhi[b]) * nl + area(rlo[b + 1], rhi[b + 1]) * nr) / parent;
                if (cost < bestCost) { bestCost = cost; bestAx = ax; bestSplit = b; }
            }
        }
        if (bestAx < 0 || bestCost >= static_cast<double>(e - s)) return false;
        const double ext = cext[bestAx];
        if (ext <= 1.0e-6) return false;
        const double pos = clo[bestAx] + ext * (static_cast<double>(bestSplit + 1) / static_cast<double>(kBins));
        const D3* cc = c.data();
        auto it = std::partition(perm.begin() + s, perm.begin() + e,
                                 [cc, bestAx, pos](int32_t t) { return cc[t][bestAx] < pos; });
        mid = static_cast<int>(it - perm.begin());
        return mid > s && mid < e;
    }
    // src/scene/bvhBuilder.cpp:250-312
    void build(int s, int e, int depth, int threads_left) {
        if (e - s <= kLeaf) {
            leaf_n[s] = e - s;
            return;
        }
        D3 lo0{kBig, kBig, kBig}, hi0{-kBig, -kBig, -kBig};
        for (int i = s; i < e; ++i) { lo0 = dmin(lo0, lo[perm[i]]); hi0 = dmax(hi0, hi[perm[i]]); }
        int mid = -1;
        bool ok = split_sah(s, e, lo0, hi0, mid);
        if (!ok) ok = split_median(s, e, mid);
        if (!ok) {
            leaf_n[s] = e - s;
            return;
        }
        if (threads_left > 1 && e - s >= 65536) {
            std::thread left([&, s, mid, depth, threads_left] { build(s, mid, depth + 1, threads_left / 2); });
            build(mid, e, depth + 1, threads_left - threads_left / 2);
            left.join();
        } else {
            build(s, mid, depth + 1, 1);
            build(mid, e, depth + 1, 1);
        }
    }
};

}  // namespace

bool has_opposed_twins(const float* xyz, const uint32_t* idx, size_t ntris) {
    // per triangle: its three vertices sorted by bit pattern, and the parity of that sort
    struct Key {
        uint32_t v[9];
        int32_t parity;
    };
    auto key_of = [&](size_t t, Key& k) {
        uint32_t p[3][3];
        for (int c = 0; c < 3; ++c) std::memcpy(p[c], xyz + 3 * (size_t)idx[3 * t + c], 12);
        int o[3] = {0, 1, 2}, swaps = 0;
        auto less = [&](int a, int b) { return std::lexicographical_compare(p[a], p[a] + 3, p[b], p[b] + 3); };
        for (int i = 1; i < 3; ++i)
            for (int j = i; j > 0 && less(o[j], o[j - 1]); --j) { std::swap(o[j], o[j - 1]); ++swaps; }
        for (int c = 0; c < 3; ++c) std::memcpy(k.v + 3 * c, p[o[c]], 12);
        const bool repeated = std::equal(k.v, k.v + 3, k.v + 3) || std::equal(k.v + 3, k.v + 6, k.v + 6);
        k.parity = repeated ? -1 : (swaps & 1);
    };
    std::vector<std::pair<uint64_t, uint32_t>> h(ntris);
    auto hash = [&](size_t b, size_t e) {
        for (size_t t = b; t < e; ++t) {
            Key k;
            key_of(t, k);
            uint64_t x = 1469598103934665603ull;  // FNV-1a over the sorted vertices
            for (int i = 0; i < 9; ++i) {
                x ^= k.v[i];
                x *= 1099511628211ull;
            }
            h[t] = {x, (uint32_t)t};
        }
    };
    const size_t nt = std::min<size_t>(std::max(1u, std::thread::hardware_concurrency()), 1 + ntris / 65536);
    std::vector<std::thread> pool;
    for (size_t k = 1; k < nt; ++k) pool.emplace_back(hash, ntris * k / nt, ntris * (k + 1) / nt);
    hash(0, ntris / nt);
    for (auto& th : pool) th.join();
    std::sort(h.begin(), h.end());
    for (size_t a = 0; a < ntris;) {
        size_t b = a + 1;
        while (b < ntris && h[b].first == h[a].first) ++b;
        for (size_t i = a; i + 1 < b; ++i) {
            Key ki;
            key_of(h[i].second, ki);
            if (ki.parity < 0) continue;
            for (size_t j = i + 1; j < b; ++j) {
                Key kj;
                key_of(h[j].second, kj);
                if (kj.parity >= 0 && kj.parity != ki.parity && std::equal(ki.v, ki.v + 9, kj.v)) return true;
            }
        }
        a = b;
    }
    return false;
}

std::vector<int32_t> reference_walk_rank(const float* xyz, const uint32_t* idx, size_t ntris, double scale,
                                         int n_threads) {
    RefTree T;
    T.c.resize(ntris);
    T.lo.resize(ntris);
    T.hi.resize(ntris);
    T.perm.resize(ntris);
    T.leaf_n.assign(ntris, 0);
    for (size_t t = 0; t < ntris; ++t) {
        D3 v[3];
        for (int k = 0; k < 3; ++k) {
            const float* p = xyz + 3 * (size_t)idx[3 * t + k];
            v[k] = {double(p[0]) * scale, double(p[1]) * scale, double(p[2]) * scale};
        }
        // (v0 + v1 + v2) / 3, component by component (src/scene/bvhBuilder.cpp:42-44)
        T.c[t] = {(v[0].x + v[1].x + v[2].x) / 3.0, (v[0].y + v[1].y + v[2].y) / 3.0,
                  (v[0].z + v[1].z + v[2].z) / 3.0};
        T.lo[t] = dmin(dmin(v[0], v[1]), v[2]);
        T.hi[t] = dmax(dmax(v[0], v[1]), v[2]);
        T.perm[t] = (int32_t)t;
    }
    const int nt = n_threads > 0 ? n_threads : (int)std::max(1u, std::thread::hardware_concurrency());
    if (ntris > 0) T.build(0, (int)ntris, 0, nt);
    // leaves right to left (the right subtree is walked first), each leaf's triangles in order
    std::vector<int32_t> rank(ntris);
    int32_t r = 0;
    size_t end = ntris;
    while (end > 0) {
        size_t s = end - 1;
        while (T.leaf_n[s] == 0) --s;
        for (size_t i = s; i < end; ++i) rank[(size_t)T.perm[i]] = r++;
        end = s;
    }
    return rank;
}

}  // namespace sbr
