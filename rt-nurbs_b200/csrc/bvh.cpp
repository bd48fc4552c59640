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
//    centroids coincide.  The partition is stable, so the tree, its leaf
//    order and its boxes depend only on the inputs, never on the order in
//    which nodes are processed: the device builder (scene_build.cu) processes
//    a level at a time and produces the same tree.
//  * collapse_to_wide: binary -> 4-wide nodes with SoA child boxes, the layout
//    the device traverses, numbered breadth-first (as the device builder
//    numbers them).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "scene_math.h"

namespace nrt {

namespace {

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
    std::vector<float> cen(prims.size() * 3);
    for (size_t i = 0; i < prims.size(); ++i)
        for (int k = 0; k < 3; ++k) cen[3 * i + k] = centre(prims[i], k);
    SahBins bins;
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
        float ext[3], scale[3];
        for (int a = 0; a < 3; ++a) {
            ext[a] = chi[a] - clo[a];
            scale[a] = kSahBins / ext[a];
            for (int k = 0; k < kSahBins; ++k) {
                bins.cnt[a][k] = 0;
                for (int c = 0; c < 3; ++c) { bins.lo[a][k][c] = INFINITY; bins.hi[a][k][c] = -INFINITY; }
            }
            if (!(ext[a] > 0)) continue;
            for (uint32_t i = first; i < first + count; ++i) {
                const int id = out.order[i];
                const int b = sah_bin(cen[3 * id + a], clo[a], scale[a]);
                ++bins.cnt[a][b];
                for (int c = 0; c < 3; ++c) {
                    bins.lo[a][b][c] = fminf(bins.lo[a][b][c], prims[id].lo[c]);
                    bins.hi[a][b][c] = fmaxf(bins.hi[a][b][c], prims[id].hi[c]);
                }
            }
        }
        int axis, split;
        sah_choose(bins, ext, axis, split);
        if (axis < 0) continue;  // all centroids coincide: keep as a leaf
        auto left_of = [&](int id) { return sah_bin(cen[3 * id + axis], clo[axis], scale[axis]) < split; };
        int32_t* beg = out.order.data() + first;
        int32_t* mid = std::stable_partition(beg, beg + count, left_of);
        const uint32_t nl = (uint32_t)(mid - beg);
        if (nl == 0 || nl == count) continue;
        const uint32_t L = out.used++, R = out.used++;
        out.left_first[L] = first; out.prim_count[L] = nl;
        out.left_first[R] = first + nl; out.prim_count[R] = count - nl;
        out.left_first[node] = L; out.prim_count[node] = 0;
        sah_sides(bins, axis, split, out.box[L], out.box[R]);
        todo.push_back(L);
        todo.push_back(R);
    }
}

void collapse_to_wide(const BinaryBVH& bin, std::vector<Node4>& out, int& depth) {
    out.clear();
    depth = 0;
    struct Item { uint32_t bin_node; int level; };
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
    // breadth first: wide node w is queue entry w, its inner children are
    // numbered in order as they are queued
    std::vector<Item> queue{{0u, 1}};
    out.emplace_back();
    blank(out[0]);
    for (size_t w = 0; w < queue.size(); ++w) {
        const Item it = queue[w];
        depth = std::max(depth, it.level);
        uint32_t kids[4];
        const int n = wide_kids(it.bin_node, bin.box.data(), bin.left_first.data(), bin.prim_count.data(), kids);
        for (int c = 0; c < n; ++c) {
            const uint32_t b = kids[c];
            if (bin.prim_count[b] > 0) {
                set_child(out[w], c, b, ~(int32_t)bin.left_first[b], (int32_t)bin.prim_count[b]);
            } else {
                const int idx = (int)out.size();
                out.emplace_back();
                blank(out.back());
                set_child(out[w], c, b, idx, 0);
                queue.push_back({b, it.level + 1});
            }
        }
    }
}

}  // namespace nrt
