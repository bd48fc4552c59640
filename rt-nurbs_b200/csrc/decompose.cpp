// decompose.cpp -- NURBS surface -> Bezier patches by knot insertion.
//
// Algorithm A5.7 of The NURBS Book (Piegl & Tiller), applied first along u to
// the whole net (giving strips of p+1 rows) and then along v to every strip,
// as BezierPatchOps::getPatch does (src/math/bezier_patch.h:86-139) with
// NurbsOps::decomposeSurface (src/math/nurbs.h:143-250).  The arithmetic is
// float with the reference's order of operations (alpha from knot ratios,
// then alpha*Q[k] + (1-alpha)*Q[k-1] per coordinate), so on degrees the
// reference supports the control points are bit-identical to getPatch's.
// Unlike the reference (NURBS_MAX_DEGREE = 4, src/constants.h:31-32) degrees
// up to NRT_MAX_DEGREE are accepted.
#include <cmath>
#include <cstring>

#include "nrt_internal.h"

namespace nrt {

namespace {

struct P4 {
    float x, y, z, w;
};

// Breakpoints of a clamped knot vector: U[p], each new interior value, U[last-p].
// (segs(), src/math/bezier_patch.h:46-53)
int spans(const float* U, int last, int p, float* out) {
    int nb = 0;
    out[nb++] = U[p];
    for (int i = p + 1; i <= last - p - 1; ++i)
        if (U[i] != U[i - 1]) out[nb++] = U[i];
    out[nb] = U[last - p];
    return nb;
}

// Strided 2D view: element (k, r) with k along the split direction.
struct View {
    P4* base;
    long sk, sr, piece;  // stride along k, across r, between pieces
    P4& at(int piece_idx, int k, int r) const { return base[piece_idx * piece + k * sk + r * sr]; }
};

// Split `lines` curves of degree `deg` (knots K[0..last]) into Bezier pieces.
int split_axis(const P4* src, long src_sk, long src_sr, int lines, int deg, const float* K, int last, View dst) {
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

}  // namespace

int check_surface(const nrt_nurbs_surface& s) {
    if (!s.control_points || !s.u_knots || !s.v_knots)
        return fail(NRT_ERR_INVALID, "surface has a null control point or knot pointer");
    if (s.p < 1 || s.q < 1 || s.p > NRT_MAX_DEGREE || s.q > NRT_MAX_DEGREE)
        return fail(NRT_ERR_INVALID, "degree (%d,%d) outside 1..%d", s.p, s.q, NRT_MAX_DEGREE);
    if (s.n < s.p || s.m < s.q) return fail(NRT_ERR_INVALID, "net (%d,%d) too small for degree (%d,%d)", s.n + 1,
                                            s.m + 1, s.p, s.q);
    const float* UV[2] = {s.u_knots, s.v_knots};
    const int last[2] = {s.n + s.p + 1, s.m + s.q + 1}, deg[2] = {s.p, s.q};
    for (int d = 0; d < 2; ++d) {
        for (int i = 0; i < last[d]; ++i)
            if (!(UV[d][i] <= UV[d][i + 1])) return fail(NRT_ERR_INVALID, "knot vector %c not non-decreasing", "uv"[d]);
        for (int i = 1; i <= deg[d]; ++i)
            if (UV[d][i] != UV[d][0] || UV[d][last[d] - i] != UV[d][last[d]])
                return fail(NRT_ERR_INVALID, "knot vector %c is not clamped", "uv"[d]);
        // interior multiplicity above the degree would make the surface discontinuous
        for (int i = deg[d] + 1, run = 1; i <= last[d] - deg[d] - 1; ++i) {
            run = (UV[d][i] == UV[d][i - 1]) ? run + 1 : 1;
            if (run > deg[d]) return fail(NRT_ERR_INVALID, "interior knot multiplicity above degree in %c", "uv"[d]);
        }
    }
    return NRT_OK;
}

int decompose_surface(const nrt_nurbs_surface& s, std::vector<float>& cp, std::vector<float>& ranges, int& nbU,
                      int& nbV) {
    if (int st = check_surface(s)) return st;
    std::vector<float> bu(s.n - s.p + 2), bv(s.m - s.q + 2);
    nbU = spans(s.u_knots, s.n + s.p + 1, s.p, bu.data());
    nbV = spans(s.v_knots, s.m + s.q + 1, s.q, bv.data());
    const int cols = s.m + 1;
    const long strip = (long)(s.p + 1) * cols, piece = (long)(s.p + 1) * (s.q + 1);
    std::vector<P4> strips((size_t)(nbU + 1) * strip);
    std::vector<P4> out((size_t)(nbU * nbV + 1) * piece);
    const P4* net = reinterpret_cast<const P4*>(s.control_points);
    // u pass over the whole net: strip b, row k (along u), column r
    split_axis(net, cols, 1, cols, s.p, s.u_knots, s.n + s.p + 1, View{strips.data(), cols, 1, strip});
    // v pass per strip: piece b, column k (along v), row r -> index r*(q+1)+k
    for (int b = 0; b < nbU; ++b)
        split_axis(strips.data() + b * strip, 1, cols, s.p + 1, s.q, s.v_knots, s.m + s.q + 1,
                   View{out.data() + (size_t)b * nbV * piece, 1, s.q + 1, piece});
    cp.resize((size_t)nbU * nbV * piece * 4);
    std::memcpy(cp.data(), out.data(), cp.size() * sizeof(float));
    ranges.resize((size_t)nbU * nbV * 4);
    for (int i = 0; i < nbU; ++i)
        for (int j = 0; j < nbV; ++j) {
            float* r = &ranges[4 * (size_t)(i * nbV + j)];
            r[0] = bu[i]; r[1] = bu[i + 1]; r[2] = bv[j]; r[3] = bv[j + 1];
        }
    return NRT_OK;
}

void patch_boxes(const PatchSet& ps, std::vector<Box3>& out) {
    out.resize(ps.count());
    for (int k = 0; k < ps.count(); ++k) {
        const int n = (ps.deg[2 * k] + 1) * (ps.deg[2 * k + 1] + 1);
        const float* c = &ps.cp[4 * (size_t)ps.off[k]];
        Box3 b{{INFINITY, INFINITY, INFINITY}, {-INFINITY, -INFINITY, -INFINITY}};
        for (int i = 0; i < n; ++i)  // BezierPatchOps::bounds, bezier_patch.h:158-165
            for (int a = 0; a < 3; ++a) {
                const float x = c[4 * i + a] / c[4 * i + 3];
                b.lo[a] = fminf(b.lo[a], x);
                b.hi[a] = fmaxf(b.hi[a], x);
            }
        out[k] = b;
    }
}

}  // namespace nrt
