// refine.cpp -- curvature-driven knot insertion before decomposition.
//
// The reference refines a surface along u, then along v
// (NurbsOps::curvatureRefinementU/V, src/math/nurbs.h:289-486, applied in
// that order by src/core/main.cpp:100-102 and src/core/benchmark.cpp:164-167).
// For every knot span [U_i, U_i+1) of a curve of degree p with control points
// P (dehomogenised), the number of knots to insert is
//     floor( C * max_j |A_j| * (U_i+1 - U_i)^1.5 / sqrt( sum_j |V_j| / p ) )
// where V_j = p (P_j - P_j-1) / (U_j+p - U_j) are the first-derivative
// control vectors of the span and A_j = (p-1) (V_j - V_j-1) / (U_j+p-1 - U_j)
// the second-derivative ones (NurbsOps::knotsToAdd, nurbs.h:254-281); the
// count of a span is the maximum over all lines of the net in that direction.
// The knots go in evenly spaced inside the span, one at a time, by Algorithm
// A5.1 of The NURBS Book (Piegl & Tiller) with r = 1 on every line.  The
// arithmetic is float in the reference's order of operations so that the
// counts (a truncated float) and the refined nets equal the reference's.
//
// Differences, decided: the reference's V pass sizes its scratch curve by the
// u-count (n+1) while filling m+1 points (nurbs.h:384-399), which overflows
// when m > n; here it is sized for the longer direction.  A count is capped at
// 2^20 knots per span (the reference converts any float to int).
#include <cmath>
#include <cstring>
#include <vector>

#include "nrt_internal.h"
#include "refine_math.h"

namespace nrt {

namespace {

using refine_math::V3;
struct Q4 {
    float x, y, z, w;
};

using refine_math::find_span;
using refine_math::multiplicity_at;

// Algorithm A5.1 with r = 1: insert u (span k, multiplicity s < p) into the
// curve Pw (np+1 points, knots UP) giving Qw (np+2 points) and UQ.
void insert_once(int np, int p, const float* UP, float u, int k, int s, float* UQ, const Q4* Pw, Q4* Qw) {
    const int mp = np + p + 1;
    Q4 R[NRT_MAX_DEGREE + 1];
    for (int i = 0; i <= k; ++i) UQ[i] = UP[i];
    UQ[k + 1] = u;
    for (int i = k + 1; i <= mp; ++i) UQ[i + 1] = UP[i];
    for (int i = 0; i <= k - p; ++i) Qw[i] = Pw[i];
    for (int i = k - s; i <= np; ++i) Qw[i + 1] = Pw[i];
    for (int i = 0; i <= p - s; ++i) R[i] = Pw[k - p + i];
    const int L = k - p + 1;
    for (int i = 0; i <= p - 1 - s; ++i) {
        const float alpha = (u - UP[L + i]) / (UP[i + k + 1] - UP[L + i]);
        const float beta = 1.0f - alpha;
        R[i] = {alpha * R[i + 1].x + beta * R[i].x, alpha * R[i + 1].y + beta * R[i].y,
                alpha * R[i + 1].z + beta * R[i].z, alpha * R[i + 1].w + beta * R[i].w};
    }
    Qw[L] = R[0];
    Qw[k - s] = R[p - 1 - s];
    for (int i = L + 1; i < k - s; ++i) Qw[i] = R[i - L];
}

// One direction.  The net is rows x cols points, row-major; the curves run
// along the rows index when along_u (one curve per column), else along the
// columns index (one curve per row).  K: knots of the refined direction.
void refine_dir(std::vector<Q4>& net, int& rows, int& cols, std::vector<float>& K, int deg, float C, bool along_u) {
    const int len = along_u ? rows : cols, lines = along_u ? cols : rows;
    const int n = len - 1;
    auto at = [&](int r, int c) -> Q4& { return net[(size_t)r * cols + c]; };
    std::vector<V3> curve(len);
    std::vector<int> add(n - deg + 1, 0);
    for (int i = deg; i <= n; ++i) {
        int ni = 0;
        for (int l = 0; l < lines; ++l) {
            for (int a = 0; a <= n; ++a) {
                const Q4& q = along_u ? at(a, l) : at(l, a);
                curve[a] = {q.x / q.w, q.y / q.w, q.z / q.w};
            }
            const V3* P = curve.data();
            ni = std::max(ni, refine_math::knot_count([P](int a) { return P[a]; }, K.data(), i, C, deg));
        }
        add[i - deg] = ni;
    }
    long total = 0;
    for (int a : add) total += a;
    if (total == 0) return;
    const int n_final = n + (int)total;
    std::vector<float> Usrc(K), Udst(n_final + deg + 2);
    Usrc.resize(n_final + deg + 2);
    // lines stored contiguously, each with room for n_final+1 points
    std::vector<Q4> src((size_t)lines * (n_final + 1)), dst(src.size());
    for (int l = 0; l < lines; ++l)
        for (int a = 0; a <= n; ++a) src[(size_t)l * (n_final + 1) + a] = along_u ? at(a, l) : at(l, a);
    int ncur = n;
    for (int i = deg; i <= n; ++i) {
        const int cnt = add[i - deg];
        const float lo = K[i], hi = K[i + 1];
        for (int j = 1; j <= cnt; ++j) {
            const float u = lo + (hi - lo) * j / (float)(cnt + 1);
            const int k = find_span(ncur, deg, u, Usrc.data());
            const int s = multiplicity_at(Usrc.data(), k, u);
            if (s >= deg) continue;  // cannot happen for distinct interior values; keeps A5.1's precondition
            for (int l = 0; l < lines; ++l)
                insert_once(ncur, deg, Usrc.data(), u, k, s, Udst.data(), &src[(size_t)l * (n_final + 1)],
                            &dst[(size_t)l * (n_final + 1)]);
            std::swap(src, dst);
            std::swap(Usrc, Udst);
            ++ncur;
        }
    }
    // write back
    if (along_u) rows = ncur + 1;
    else cols = ncur + 1;
    net.assign((size_t)rows * cols, Q4{});
    for (int l = 0; l < lines; ++l)
        for (int a = 0; a <= ncur; ++a) {
            const Q4& q = src[(size_t)l * (n_final + 1) + a];
            if (along_u) net[(size_t)a * cols + l] = q;
            else net[(size_t)l * cols + a] = q;
        }
    K.assign(Usrc.begin(), Usrc.begin() + ncur + deg + 2);
}

int refine(const nrt_nurbs_surface& s, float C, std::vector<Q4>& net, std::vector<float>& U, std::vector<float>& V,
           int& n, int& m) {
    if (int st = check_surface(s)) return st;
    n = s.n;
    m = s.m;
    net.resize((size_t)(n + 1) * (m + 1));
    std::memcpy(net.data(), s.control_points, net.size() * sizeof(Q4));
    U.assign(s.u_knots, s.u_knots + n + s.p + 2);
    V.assign(s.v_knots, s.v_knots + m + s.q + 2);
    if (!(C > 0.f)) return NRT_OK;
    int rows = n + 1, cols = m + 1;
    refine_dir(net, rows, cols, U, s.p, C, true);
    refine_dir(net, rows, cols, V, s.q, C, false);
    n = rows - 1;
    m = cols - 1;
    return NRT_OK;
}

}  // namespace

}  // namespace nrt

extern "C" {

int nrt_refine_count(const nrt_nurbs_surface* surf, float C, int* n_out, int* m_out) {
    if (!surf || !n_out || !m_out) return nrt::fail(NRT_ERR_INVALID, "null argument");
    std::vector<nrt::Q4> net;
    std::vector<float> U, V;
    int n = 0, m = 0;
    if (int st = nrt::refine(*surf, C, net, U, V, n, m)) return st;
    *n_out = n;
    *m_out = m;
    return NRT_OK;
}

int nrt_refine_surface(const nrt_nurbs_surface* surf, float C, float* cp_out, float* u_knots_out, float* v_knots_out,
                       int* n_out, int* m_out) {
    if (!surf || !cp_out || !u_knots_out || !v_knots_out || !n_out || !m_out)
        return nrt::fail(NRT_ERR_INVALID, "null argument");
    std::vector<nrt::Q4> net;
    std::vector<float> U, V;
    int n = 0, m = 0;
    if (int st = nrt::refine(*surf, C, net, U, V, n, m)) return st;
    std::memcpy(cp_out, net.data(), net.size() * sizeof(nrt::Q4));
    std::memcpy(u_knots_out, U.data(), U.size() * sizeof(float));
    std::memcpy(v_knots_out, V.data(), V.size() * sizeof(float));
    *n_out = n;
    *m_out = m;
    return NRT_OK;
}

}  // extern "C"
