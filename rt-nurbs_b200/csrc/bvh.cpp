// bvh.cpp -- bounding volume hierarchies over patch boxes.
//
//  * build_exact_sah: the reference's builder (BvhOps::buildBVH / subdivide /
//    evaluateSAH / updateNodeBounds, src/core/bvh.h:47-179): every primitive
//    centroid on every axis is a split candidate, cost = nL*halfArea(L) +
//    nR*halfArea(R), Hoare-style partition, recursion until a split leaves
//    one side empty.  O(N^2) per level; kept for node-for-node parity on small
//    scenes.
//  * build_binned_sah: 32-bin SAH (same cost function), O(N log N), used for
//    scenes.  Splits until a node holds at most max_leaf patches or its
//    centroids coincide.
//  * collapse_to_wide: binary -> 4-wide nodes with SoA child boxes, the layout
//    the device traverses.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "nrt_internal.h"

namespace nrt {

namespace {

inline Box3 empty_box() { return {{INFINITY, INFINITY, INFINITY}, {-INFINITY, -INFINITY, -INFINITY}}; }
inline Box3 join(const Box3& a, const Box3& b) {
    Box3 r;
    for (int k = 0; k < 3; ++k) {
        r.lo[k] = fminf(a.lo[k], b.lo[k]);
        r.hi[k] = fmaxf(a.hi[k], b.hi[k]);
    }
    return r;
}
inline float centre(const Box3& b, int k) { return .5f * (b.lo[k] + b.hi[k]); }
inline float half_area(const Box3& b) {  // bounds_ops.h:72-77
    const float ex = b.hi[0] - b.lo[0], ey = b.hi[1] - b.lo[1], ez = b.hi[2] - b.lo[2];
    return ex * ey + ey * ez + ez * ex;
}

struct ExactBuilder {
    const std::vector<Box3>& prim;
    BinaryBVH& out;

    float cost(uint32_t first, uint32_t count, int axis, float pos) const {
        Box3 l = empty_box(), r = empty_box();
        int nl = 0, nr = 0;
        for (uint32_t i = first; i < first + count; ++i) {
            const Box3& b = prim[out.order[i]];
            if (centre(b, axis) < pos) { ++nl; l = join(l, b); }
            else { ++nr; r = join(r, b); }
        }
        const float c = nl * half_area(l) + nr * half_area(r);
        return c > 0 ? c : 1e30f;
    }
    void fit(uint32_t node) {
        Box3 b = empty_box();
        for (uint32_t i = out.left_first[node]; i < out.left_first[node] + out.prim_count[node]; ++i)
            b = join(b, prim[out.order[i]]);
        out.box[node] = b;
    }
    void split(uint32_t node) {
        const uint32_t first = out.left_first[node], count = out.prim_count[node];
        int axis = 1;
        float pos = 0, best = 1e30f;
        for (int a = 0; a < 3; ++a)
            for (uint32_t i = first; i < first + count; ++i) {
                const float cand = centre(prim[out.order[i]], a);
                const float c = cost(first, count, a, cand);
                if (c < best) { best = c; pos = cand; axis = a; }
            }
        int i = (int)first, j = (int)(first + count) - 1;
        while (i <= j) {
            if (centre(prim[out.order[i]], axis) < pos) ++i;
            else std::swap(out.order[i], out.order[j--]);
        }
        const uint32_t nl = (uint32_t)i - first;
        if (nl == 0 || nl == count) return;
        const uint32_t L = out.used++, R = out.used++;
        out.left_first[L] = first; out.prim_count[L] = nl;
        out.left_first[R] = (uint32_t)i; out.prim_count[R] = count - nl;
        out.left_first[node] = L; out.prim_count[node] = 0;
        fit(L); fit(R);
        split(L); split(R);
    }
};

void init_out(const std::vector<Box3>& prims, BinaryBVH& out) {
    const size_t N = prims.size();
    const size_t M = N ? 2 * N - 1 : 1;
    out.box.assign(M, Box3{{0, 0, 0}, {0, 0, 0}});
    out.left_first.assign(M, 0);
    out.prim_count.assign(M, 0);
    out.order.resize(N);
    Box3 root = empty_box();
    for (size_t i = 0; i < N; ++i) { out.order[i] = (int32_t)i; root = join(root, prims[i]); }
    out.box[0] = root;
    out.left_first[0] = 0;
    out.prim_count[0] = (uint32_t)N;
    out.used = 1;
}

}  // namespace

void build_exact_sah(const std::vector<Box3>& prims, BinaryBVH& out) {
    init_out(prims, out);
    if (prims.empty()) return;
    ExactBuilder b{prims, out};
    b.split(0);
}

void build_binned_sah(const std::vector<Box3>& prims, int max_leaf, BinaryBVH& out) {
    init_out(prims, out);
    if (prims.empty()) return;
    constexpr int BINS = 32;
    std::vector<float> cen(prims.size() * 3);
    for (size_t i = 0; i < prims.size(); ++i)
        for (int k = 0; k < 3; ++k) cen[3 * i + k] = centre(prims[i], k);
    // explicit stack instead of recursion (depth is unbounded for bad inputs)
    std::vector<uint32_t> todo{0};
    while (!todo.empty()) {
        const uint32_t node = todo.back();
        todo.pop_back();
        const uint32_t first = out.left_first[node], count = out.prim_count[node];
        if ((int)count <= max_leaf) continue;
        float clo[3] = {INFINITY, INFINITY, INFINITY}, chi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (uint32_t i = first; i < first + count; ++i)
            for (int k = 0; k < 3; ++k) {
                clo[k] = fminf(clo[k], cen[3 * out.order[i] + k]);
                chi[k] = fmaxf(chi[k], cen[3 * out.order[i] + k]);
            }
        int best_axis = -1, best_split = 0;
        float best_cost = INFINITY;
        for (int a = 0; a < 3; ++a) {
            const float ext = chi[a] - clo[a];
            if (!(ext > 0)) continue;
            Box3 bb[BINS];
            int bc[BINS] = {0};
            for (int k = 0; k < BINS; ++k) bb[k] = empty_box();
            const float scale = BINS / ext;
            for (uint32_t i = first; i < first + count; ++i) {
                const int id = out.order[i];
                int b = (int)((cen[3 * id + a] - clo[a]) * scale);
                b = std::min(std::max(b, 0), BINS - 1);
                ++bc[b];
                bb[b] = join(bb[b], prims[id]);
            }
            float right_area[BINS];
            int right_count[BINS];
            Box3 acc = empty_box();
            int n = 0;
            for (int k = BINS - 1; k > 0; --k) {
                acc = join(acc, bb[k]);
                n += bc[k];
                right_area[k] = half_area(acc);
                right_count[k] = n;
            }
            acc = empty_box();
            n = 0;
            for (int k = 0; k < BINS - 1; ++k) {
                acc = join(acc, bb[k]);
                n += bc[k];
                if (n == 0 || right_count[k + 1] == 0) continue;
                const float c = n * half_area(acc) + right_count[k + 1] * right_area[k + 1];
                if (c < best_cost) { best_cost = c; best_axis = a; best_split = k + 1; }
            }
        }
        if (best_axis < 0) continue;  // all centroids coincide: keep as a leaf
        const float ext = chi[best_axis] - clo[best_axis], scale = BINS / ext;
        auto left_of = [&](int id) {
            int b = (int)((cen[3 * id + best_axis] - clo[best_axis]) * scale);
            b = std::min(std::max(b, 0), BINS - 1);
            return b < best_split;
        };
        int32_t* beg = out.order.data() + first;
        int32_t* mid = std::partition(beg, beg + count, left_of);
        const uint32_t nl = (uint32_t)(mid - beg);
        if (nl == 0 || nl == count) continue;
        const uint32_t L = out.used++, R = out.used++;
        out.left_first[L] = first; out.prim_count[L] = nl;
        out.left_first[R] = first + nl; out.prim_count[R] = count - nl;
        out.left_first[node] = L; out.prim_count[node] = 0;
        for (uint32_t c : {L, R}) {
            Box3 b = empty_box();
            for (uint32_t i = out.left_first[c]; i < out.left_first[c] + out.prim_count[c]; ++i)
                b = join(b, prims[out.order[i]]);
            out.box[c] = b;
            todo.push_back(c);
        }
    }
}

void collapse_to_wide(const BinaryBVH& bin, std::vector<Node4>& out, int& depth) {
    out.clear();
    depth = 0;
    struct Item { uint32_t bin_node; int wide_index; int level; };
    auto set_child = [&](Node4& n, int c, uint32_t bnode, int32_t ref, int32_t cnt) {
        const Box3& b = bin.box[bnode];
        n.lo_x[c] = b.lo[0]; n.lo_y[c] = b.lo[1]; n.lo_z[c] = b.lo[2];
        n.hi_x[c] = b.hi[0]; n.hi_y[c] = b.hi[1]; n.hi_z[c] = b.hi[2];
        n.child[c] = ref;
        n.count[c] = cnt;
    };
    auto blank = [](Node4& n) {
        for (int c = 0; c < 4; ++c) {
            n.lo_x[c] = n.lo_y[c] = n.lo_z[c] = INFINITY;
            n.hi_x[c] = n.hi_y[c] = n.hi_z[c] = -INFINITY;
            n.child[c] = -1;
            n.count[c] = 0;
        }
    };
    out.emplace_back();
    blank(out[0]);
    std::vector<Item> todo{{0u, 0, 1}};
    while (!todo.empty()) {
        Item it = todo.back();
        todo.pop_back();
        depth = std::max(depth, it.level);
        // gather up to 4 children by opening the largest inner child repeatedly
        std::vector<uint32_t> kids;
        if (bin.prim_count[it.bin_node] > 0) kids.push_back(it.bin_node);  // the root itself is a leaf
        else { kids.push_back(bin.left_first[it.bin_node]); kids.push_back(bin.left_first[it.bin_node] + 1); }
        while (kids.size() < 4) {
            int pick = -1;
            float best = -1;
            for (size_t k = 0; k < kids.size(); ++k)
                if (bin.prim_count[kids[k]] == 0) {
                    const float a = half_area(bin.box[kids[k]]);
                    if (a > best) { best = a; pick = (int)k; }
                }
            if (pick < 0) break;
            const uint32_t b = kids[pick];
            kids.erase(kids.begin() + pick);
            kids.push_back(bin.left_first[b]);
            kids.push_back(bin.left_first[b] + 1);
        }
        for (size_t c = 0; c < kids.size(); ++c) {
            const uint32_t b = kids[c];
            if (bin.prim_count[b] > 0) {
                set_child(out[it.wide_index], (int)c, b, ~(int32_t)bin.left_first[b], (int32_t)bin.prim_count[b]);
            } else {
                const int idx = (int)out.size();
                out.emplace_back();
                blank(out.back());
                set_child(out[it.wide_index], (int)c, b, idx, 0);
                todo.push_back({b, idx, it.level + 1});
            }
        }
    }
}

}  // namespace nrt
