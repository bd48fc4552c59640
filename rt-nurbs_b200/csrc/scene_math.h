// scene_math.h -- the scene build's arithmetic, shared by the host builder
// (decompose.cpp, bvh.cpp) and the device builder (scene_build.cu), so that
// both produce the same bits.  Every function here is plain float/int code
// with one rounding per operation: the host side is compiled with
// -ffp-contract=off and the device side with -fmad=false, and the divisions
// and square roots used are the correctly rounded ones on both.
#pragma once

#include <cmath>
#include <cstdint>

#include "nrt_internal.h"

#ifdef __CUDACC__
#define NRT_HD __host__ __device__
#else
#define NRT_HD
#endif

namespace nrt {

// ---------------------------------------------------------------------------
// Boxes (bounds_ops.h: boundUnion :48-59, centroid :39-45, bound_area :72-77)

NRT_HD inline Box3 empty_box() { return {{INFINITY, INFINITY, INFINITY}, {-INFINITY, -INFINITY, -INFINITY}}; }
NRT_HD inline Box3 join(const Box3& a, const Box3& b) {
    Box3 r;
    for (int k = 0; k < 3; ++k) {
        r.lo[k] = fminf(a.lo[k], b.lo[k]);
        r.hi[k] = fmaxf(a.hi[k], b.hi[k]);
    }
    return r;
}
NRT_HD inline float centre(const Box3& b, int k) { return .5f * (b.lo[k] + b.hi[k]); }
NRT_HD inline float half_area(const Box3& b) {
    const float ex = b.hi[0] - b.lo[0], ey = b.hi[1] - b.lo[1], ez = b.hi[2] - b.lo[2];
    return ex * ey + ey * ez + ez * ex;
}

// Box of a patch's dehomogenised control points (BezierPatchOps::bounds,
// src/math/bezier_patch.h:153-169); P holds n weighted-homogeneous points.
NRT_HD inline Box3 patch_box(const float* P, int n) {
    Box3 b = empty_box();
    for (int i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) {
            const float x = P[4 * i + a] / P[4 * i + 3];
            b.lo[a] = fminf(b.lo[a], x);
            b.hi[a] = fmaxf(b.hi[a], x);
        }
    return b;
}

// ---------------------------------------------------------------------------
// Binned SAH (32 bins per axis, cost nL*halfArea(L) + nR*halfArea(R), the
// reference's cost function, src/core/bvh.h:47-69)

constexpr int kSahBins = 32;

// Bin of a centroid coordinate c in a node whose centroids start at lo, with
// scale = kSahBins / extent.  NaN lands in bin 0, +inf in the last bin.
NRT_HD inline int sah_bin(float c, float lo, float scale) {
    const float f = (c - lo) * scale;
    return f >= 0.f ? (f < (float)kSahBins ? (int)f : kSahBins - 1) : 0;
}

// Bins of one node, all three axes: bin box lo/hi [axis][bin][xyz] and counts.
struct SahBins {
    float lo[3][kSahBins][3];
    float hi[3][kSahBins][3];
    int cnt[3][kSahBins];
};

// The split of a node from its bins: the axis and first right bin of the
// cheapest split over axes with a positive centroid extent (ties keep the
// earlier axis and bin), or axis -1 when no axis splits.
NRT_HD inline void sah_choose(const SahBins& B, const float ext[3], int& best_axis, int& best_split) {
    best_axis = -1;
    best_split = 0;
    float best_cost = INFINITY;
    for (int a = 0; a < 3; ++a) {
        if (!(ext[a] > 0)) continue;
        float right_area[kSahBins];
        int right_count[kSahBins];
        Box3 acc = empty_box();
        int n = 0;
        for (int k = kSahBins - 1; k > 0; --k) {
            const Box3 bk = {{B.lo[a][k][0], B.lo[a][k][1], B.lo[a][k][2]}, {B.hi[a][k][0], B.hi[a][k][1], B.hi[a][k][2]}};
            acc = join(acc, bk);
            n += B.cnt[a][k];
            right_area[k] = half_area(acc);
            right_count[k] = n;
        }
        acc = empty_box();
        n = 0;
        for (int k = 0; k < kSahBins - 1; ++k) {
            const Box3 bk = {{B.lo[a][k][0], B.lo[a][k][1], B.lo[a][k][2]}, {B.hi[a][k][0], B.hi[a][k][1], B.hi[a][k][2]}};
            acc = join(acc, bk);
            n += B.cnt[a][k];
            if (n == 0 || right_count[k + 1] == 0) continue;
            const float c = n * half_area(acc) + right_count[k + 1] * right_area[k + 1];
            if (c < best_cost) { best_cost = c; best_axis = a; best_split = k + 1; }
        }
    }
}

// The boxes of the two sides of a split, joined from the bins.
NRT_HD inline void sah_sides(const SahBins& B, int axis, int split, Box3& left, Box3& right) {
    left = empty_box();
    right = empty_box();
    for (int k = 0; k < kSahBins; ++k) {
        const Box3 bk = {{B.lo[axis][k][0], B.lo[axis][k][1], B.lo[axis][k][2]},
                         {B.hi[axis][k][0], B.hi[axis][k][1], B.hi[axis][k][2]}};
        if (k < split) left = join(left, bk);
        else right = join(right, bk);
    }
}

// ---------------------------------------------------------------------------
// Binary -> 4-wide: the children a wide node takes for binary node `node`.
// A leaf root is its own single child; otherwise start from the two children
// and open the inner child of largest half area (first on ties) until there
// are four.  Returns the number of children written to kids.
NRT_HD inline int wide_kids(uint32_t node, const Box3* box, const uint32_t* left_first, const uint32_t* prim_count,
                            uint32_t kids[4]) {
    int n = 0;
    if (prim_count[node] > 0) {
        kids[n++] = node;
        return n;
    }
    kids[n++] = left_first[node];
    kids[n++] = left_first[node] + 1;
    while (n < 4) {
        int pick = -1;
        float best = -1;
        for (int k = 0; k < n; ++k)
            if (prim_count[kids[k]] == 0) {
                const float a = half_area(box[kids[k]]);
                if (a > best) { best = a; pick = k; }
            }
        if (pick < 0) break;
        const uint32_t b = kids[pick];
        for (int k = pick; k + 1 < n; ++k) kids[k] = kids[k + 1];
        kids[n - 1] = left_first[b];
        kids[n++] = left_first[b] + 1;
    }
    return n;
}

// ---------------------------------------------------------------------------
// Breakpoints of a clamped knot vector U[0..last] of degree p: U[p], each new
// interior value, U[last-p]; returns the number of spans (segs(),
// src/math/bezier_patch.h:46-53).
NRT_HD inline int knot_spans(const float* U, int last, int p, float* out) {
    int nb = 0;
    out[nb++] = U[p];
    for (int i = p + 1; i <= last - p - 1; ++i)
        if (U[i] != U[i - 1]) out[nb++] = U[i];
    out[nb] = U[last - p];
    return nb;
}

// ---------------------------------------------------------------------------
// Knot-insertion decomposition, Algorithm A5.7 of The NURBS Book (Piegl &
// Tiller), one direction; NurbsOps::decomposeSurface, src/math/nurbs.h:143-250.

struct P4 {
    float x, y, z, w;
};

// Strided 2D view: element (k, r) of piece `piece_idx`, k along the split direction.
struct View {
    P4* base;
    long sk, sr, piece;  // stride along k, across r, between pieces
    NRT_HD P4& at(int piece_idx, int k, int r) const { return base[piece_idx * piece + k * sk + r * sr]; }
};

// Split `lines` curves of degree `deg` (knots K[0..last]) into Bezier pieces;
// returns the number of pieces.  Each line's arithmetic is independent of the
// others, so one call over many lines and many calls over one line each give
// the same points.
NRT_HD inline int split_axis(const P4* src, long src_sk, long src_sr, int lines, int deg, const float* K, int last,
                             View dst) {
    float alpha[NRT_MAX_DEGREE + 1];
    int a = deg, b = deg + 1, nb = 0;
    for (int k = 0; k <= deg; ++k)
        for (int r = 0; r < lines; ++r) dst.at(0, k, r) = src[k * src_sk + r * src_sr];
    while (b < last) {
        const int first = b;
        while (b < last && K[b + 1] == K[b]) ++b;
        const int mult = b - first + 1;
        if (mult < deg) {
            const float numer = K[b] - K[a];
            for (int j = deg; j > mult; --j) alpha[j - mult - 1] = numer / (K[a + j] - K[a]);
            const int inserts = deg - mult;
            for (int j = 1; j <= inserts; ++j) {
                const int s = mult + j;
                for (int k = deg; k >= s; --k) {
                    const float al = alpha[k - s], be = 1.0f - al;
                    for (int r = 0; r < lines; ++r) {
                        P4& cur = dst.at(nb, k, r);
                        const P4& prev = dst.at(nb, k - 1, r);
                        cur.x = al * cur.x + be * prev.x;
                        cur.y = al * cur.y + be * prev.y;
                        cur.z = al * cur.z + be * prev.z;
                        cur.w = al * cur.w + be * prev.w;
                    }
                }
                if (b < last)  // the next piece starts with this one's last points
                    for (int r = 0; r < lines; ++r) dst.at(nb + 1, inserts - j, r) = dst.at(nb, deg, r);
            }
        }
        ++nb;
        if (b < last) {
            for (int k = deg - mult; k <= deg; ++k)
                for (int r = 0; r < lines; ++r) dst.at(nb, k, r) = src[(b - deg + k) * src_sk + r * src_sr];
            a = b;
            ++b;
        }
    }
    return nb;
}

}  // namespace nrt
