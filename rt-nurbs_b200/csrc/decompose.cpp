// decompose.cpp -- NURBS surface -> Bezier patches by knot insertion.
//
// Algorithm A5.7 of The NURBS Book (Piegl & Tiller), applied first along u to
// the whole net (giving strips of p+1 rows) and then along v to every strip,
// as BezierPatchOps::getPatch does (src/math/bezier_patch.h:86-139) with
// NurbsOps::decomposeSurface (src/math/nurbs.h:143-250).  The arithmetic is
// float with the reference's order of operations (alpha from knot ratios,
// then alpha*Q[k] + (1-alpha)*Q[k-1] per coordinate), so on degrees the
// reference supports the control points are bit-identical to getPatch's.
// The per-line step (split_axis) lives in scene_math.h, shared with the
// device builder.
// Unlike the reference (NURBS_MAX_DEGREE = 4, src/constants.h:31-32) degrees
// up to NRT_MAX_DEGREE are accepted.
#include <cmath>
#include <cstring>

#include "scene_math.h"

namespace nrt {

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
    nbU = knot_spans(s.u_knots, s.n + s.p + 1, s.p, bu.data());
    nbV = knot_spans(s.v_knots, s.m + s.q + 1, s.q, bv.data());
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
    for (int k = 0; k < ps.count(); ++k)
        out[k] = patch_box(&ps.cp[4 * (size_t)ps.off[k]], (ps.deg[2 * k] + 1) * (ps.deg[2 * k + 1] + 1));
}

}  // namespace nrt
