// oracle.cpp -- CPU restatement of the rt-nurbs intersection path.
//
// TEST INFRASTRUCTURE ONLY.  Nothing in the product library links or calls this
// file; only tests/, the smoke check and bench.py's CPU-baseline leg load it,
// and only as the checker (or the timed CPU baseline), never as the product.
//
// Every function restates one piece of Frostbite16/rt-nurbs and cites the file
// and line it follows (paths are relative to the reference project root).  The
// float instantiation keeps the reference's order of floating-point operations
// so that, compiled with -ffp-contract=off, it reproduces the reference's host
// build bit for bit; the double instantiation is the FP64 oracle that the CUDA
// results are judged against.
//
// Build: see oracle/Makefile (g++ -O2 -fopenmp -ffp-contract=off -shared).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <type_traits>
#include <vector>

namespace orc {

template <class T> struct V3 { T x, y, z; };
template <class T> struct V4 { T x, y, z, w; };

template <class T> static inline V3<T> sub3(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> static inline V3<T> scale3(V3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> static inline T dot3(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> static inline V3<T> cross3(V3<T> a, V3<T> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T> static inline V4<T> sub4(V4<T> a, V4<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w}; }
template <class T> static inline V4<T> scale4(V4<T> a, T s) { return {a.x * s, a.y * s, a.z * s, a.w * s}; }
// (1-t)*a + t*b, evaluated as the reference's de Casteljau step
// (src/math/bezier_patch.h:63): scale both, then add.
template <class T> static inline V4<T> mix4(V4<T> a, V4<T> b, T t) {
    T s = T(1) - t;
    return {a.x * s + b.x * t, a.y * s + b.y * t, a.z * s + b.z * t, a.w * s + b.w * t};
}
template <class T> static inline V3<T> dehom(V4<T> c) {
    T iw = T(1) / c.w;  // src/math/bezier_patch.h:33-35
    return {c.x * iw, c.y * iw, c.z * iw};
}

// ---------------------------------------------------------------------------
// Knot breakpoints: first knot p, each distinct interior knot, last knot.
// Follows segs(), src/math/bezier_patch.h:46-53.
static int breakpoints(const float* U, int last, int p, float* out) {
    int nb = 0;
    out[nb++] = U[p];
    for (int i = p + 1; i <= last - p - 1; ++i)
        if (U[i] != U[i - 1]) out[nb++] = U[i];
    out[nb] = U[last - p];
    return nb;
}

// ---------------------------------------------------------------------------
// Algorithm A5.7 (The NURBS Book, Piegl & Tiller): split a surface into Bezier
// strips along one direction by knot insertion.  Restates
// NurbsOps::decomposeSurface, src/math/nurbs.h:143-250.
//
//  dir 0 (U, nurbs.h:152-198):  P is (n+1) x (m+1), row stride m+1; the output
//      strip b holds (p+1) x (m+1) points at Q[b*(p+1)*(m+1) + i*(m+1) + r].
//  dir 1 (V, nurbs.h:199-245):  P is (n+1) x (m+1) read with row stride m+1;
//      output piece b holds (n+1) x (q+1) at Q[b*(n+1)*(q+1) + r*(q+1) + j].
template <class T>
static int split_bezier(int n, int p, const float* U, int m, int q, const float* V, int dir,
                        const V4<T>* P, V4<T>* Q) {
    const int deg = dir == 0 ? p : q;
    const float* K = dir == 0 ? U : V;
    const int last = dir == 0 ? n + p + 1 : m + q + 1;
    const int lines = dir == 0 ? m + 1 : n + 1;  // points per "column" of the pass
    const int in_stride = m + 1;
    const int piece = dir == 0 ? (p + 1) * (m + 1) : (n + 1) * (q + 1);
    // Accessors: k = index along the split direction, r = index across it.
    auto src = [&](int k, int r) -> const V4<T>& {
        return dir == 0 ? P[k * in_stride + r] : P[r * in_stride + k];
    };
    auto dst = [&](int b, int k, int r) -> V4<T>& {
        return dir == 0 ? Q[b * piece + k * (m + 1) + r] : Q[b * piece + r * (q + 1) + k];
    };
    T alpha_tab[16];
    int nb = 0;
    int a = deg, b = deg + 1;
    for (int k = 0; k <= deg; ++k)
        for (int r = 0; r < lines; ++r) dst(0, k, r) = src(k, r);
    while (b < last) {
        const int first = b;
        while (b < last && K[b + 1] == K[b]) ++b;
        const int mult = b - first + 1;
        if (mult < deg) {
            // knot differences are exact in double, so T = double keeps full precision
            const T numer = T(K[b]) - T(K[a]);
            for (int j = deg; j > mult; --j) alpha_tab[j - mult - 1] = numer / (T(K[a + j]) - T(K[a]));
            const int ins = deg - mult;
            for (int j = 1; j <= ins; ++j) {
                const int save = ins - j, s = mult + j;
                for (int k = deg; k >= s; --k) {
                    const T al = alpha_tab[k - s];
                    const T om = T(1) - al;
                    for (int r = 0; r < lines; ++r) {
                        V4<T>& hi = dst(nb, k, r);
                        const V4<T>& lo = dst(nb, k - 1, r);
                        // alpha*Q[k] + (1-alpha)*Q[k-1]  (nurbs.h:181-182, :228-229)
                        hi = {al * hi.x + om * lo.x, al * hi.y + om * lo.y, al * hi.z + om * lo.z,
                              al * hi.w + om * lo.w};
                    }
                }
                if (b < last)
                    for (int r = 0; r < lines; ++r) dst(nb + 1, save, r) = dst(nb, deg, r);
            }
        }
        ++nb;
        if (b < last) {
            for (int k = deg - mult; k <= deg; ++k)
                for (int r = 0; r < lines; ++r) dst(nb, k, r) = src(b - deg + k, r);
            a = b;
            ++b;
        }
    }
    return nb;
}

// Patch bounding box from the dehomogenised control points (convex hull),
// BezierPatchOps::bounds, src/math/bezier_patch.h:153-169.
static void patch_box(const float* cp4, int count, float* box6) {
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = 0; i < count; ++i) {
        const float* c = cp4 + 4 * i;
        for (int k = 0; k < 3; ++k) {
            lo[k] = fminf(lo[k], c[k] / c[3]);
            hi[k] = fmaxf(hi[k], c[k] / c[3]);
        }
    }
    box6[0] = lo[0]; box6[1] = lo[1]; box6[2] = lo[2];
    box6[3] = hi[0]; box6[4] = hi[1]; box6[5] = hi[2];
}

// ---------------------------------------------------------------------------
// Exhaustive binary SAH BVH, BvhOps::buildBVH/subdivide/evaluateSAH/
// updateNodeBounds, src/core/bvh.h:47-179.  Node bounds are 6 floats
// (min xyz, max xyz, as MathExtra::bounds3f), left_first/prim_count as BVHNode.
struct Box { float lo[3], hi[3]; };
static inline Box box_empty() { return {{INFINITY, INFINITY, INFINITY}, {-INFINITY, -INFINITY, -INFINITY}}; }
static inline Box box_join(const Box& a, const Box& b) {
    Box r;
    for (int k = 0; k < 3; ++k) { r.lo[k] = fminf(a.lo[k], b.lo[k]); r.hi[k] = fmaxf(a.hi[k], b.hi[k]); }
    return r;
}
static inline float box_centre(const Box& b, int k) { return .5f * (b.lo[k] + b.hi[k]); }  // bounds_ops.h:39-45
static inline float box_half_area(const Box& b) {  // bounds_ops.h:72-77
    float ex = b.hi[0] - b.lo[0], ey = b.hi[1] - b.lo[1], ez = b.hi[2] - b.lo[2];
    return ex * ey + ey * ez + ez * ex;
}

struct SahBuilder {
    const Box* prim;
    std::vector<uint32_t> order;
    Box* node_box;
    uint32_t* lf;
    uint32_t* cnt;
    int used;

    float split_cost(uint32_t first, uint32_t count, int axis, float pos) const {
        Box l = box_empty(), r = box_empty();
        int nl = 0, nr = 0;
        for (uint32_t i = 0; i < count; ++i) {
            const Box& b = prim[order[first + i]];
            if (box_centre(b, axis) < pos) { ++nl; l = box_join(l, b); }
            else { ++nr; r = box_join(r, b); }
        }
        float c = nl * box_half_area(l) + nr * box_half_area(r);
        return c > 0 ? c : 1e30f;
    }
    void refit(uint32_t node) {
        Box b = box_empty();
        for (uint32_t i = lf[node]; i < lf[node] + cnt[node]; ++i) b = box_join(b, prim[order[i]]);
        node_box[node] = b;
    }
    void split(uint32_t node) {
        const uint32_t first = lf[node], count = cnt[node];
        int best_axis = 1;
        float best_pos = 0, best_cost = 1e30f;
        for (int axis = 0; axis < 3; ++axis)
            for (uint32_t i = 0; i < count; ++i) {
                float pos = box_centre(prim[order[first + i]], axis);
                float c = split_cost(first, count, axis, pos);
                if (c < best_cost) { best_pos = pos; best_axis = axis; best_cost = c; }
            }
        int i = (int)first, j = (int)(first + count) - 1;
        while (i <= j) {  // Hoare-style partition, bvh.h:108-122
            if (box_centre(prim[order[i]], best_axis) < best_pos) ++i;
            else { std::swap(order[i], order[j]); --j; }
        }
        const uint32_t nleft = (uint32_t)i - first;
        if (nleft == 0 || nleft == count) return;
        const uint32_t L = used++, R = used++;
        lf[L] = first; cnt[L] = nleft;
        lf[R] = (uint32_t)i; cnt[R] = count - nleft;
        lf[node] = L; cnt[node] = 0;
        refit(L); refit(R);
        split(L); split(R);
    }
};

// ---------------------------------------------------------------------------
// The ray as two planes, MathUtils::getRayPlanes, src/math/math_utils.h:33-54.
template <class T> struct Planes { V3<T> n1, n2; T d1, d2; };

template <class T> static Planes<T> ray_planes(V3<T> o, V3<T> d) {
    const T ax = std::fabs(d.x), ay = std::fabs(d.y), az = std::fabs(d.z);
    const bool xdom = (ax > ay) && (ax > az);
    V3<T> base = xdom ? V3<T>{d.x, d.y, T(0)} : V3<T>{d.y, d.z, T(0)};
    const T rl = T(1) / std::sqrt(base.x * base.x + base.y * base.y + base.z * base.z);
    V3<T> n1 = xdom ? scale3(V3<T>{d.y, -d.x, T(0)}, rl) : scale3(V3<T>{T(0), d.z, -d.y}, rl);
    const T inv_len = T(1) / std::sqrt(d.x * d.x + d.y * d.y + d.z * d.z);
    V3<T> n2 = cross3(n1, scale3(d, inv_len));
    return {n1, n2, -dot3(n1, o), -dot3(n2, o)};
}

// Slab test returning the entry distance or +inf; tmin starts at 0.
// BoundsOps::intersectBound, src/math/bounds_ops.h:83-114.
static inline float slab(const float* b, const float* o, const float* rd) {
    float t0x = (b[0] - o[0]) * rd[0], t1x = (b[3] - o[0]) * rd[0];
    float t0y = (b[1] - o[1]) * rd[1], t1y = (b[4] - o[1]) * rd[1];
    float t0z = (b[2] - o[2]) * rd[2], t1z = (b[5] - o[2]) * rd[2];
    float lo = fmaxf(fminf(t0z, t1z), fmaxf(fminf(t0y, t1y), fmaxf(fminf(t0x, t1x), 0.0f)));
    float hi = fminf(fmaxf(t0z, t1z), fminf(fmaxf(t0y, t1y), fminf(fmaxf(t0x, t1x), INFINITY)));
    return (lo <= hi && hi > 0) ? lo : INFINITY;
}

// ---------------------------------------------------------------------------
// de Casteljau evaluation (Algorithm A1.5), src/math/bezier_patch.h:56-80.
template <class T> static V4<T> curve_point(const V4<T>* P, int n, T u) {
    V4<T> Q[8];
    for (int i = 0; i <= n; ++i) Q[i] = P[i];
    for (int k = 1; k <= n; ++k)
        for (int i = 0; i <= n - k; ++i) Q[i] = mix4(Q[i], Q[i + 1], u);
    return Q[0];
}
// Derivative via the hodograph n*(P[i+1]-P[i]).  The reference's loop also
// updates one slot past the hodograph (bezier_patch.h:76-78); that slot never
// reaches Q[0], so the tighter bound here gives the same Q[0].
template <class T> static V4<T> curve_deriv(const V4<T>* P, int n, T u) {
    if (n == 0) return {T(0), T(0), T(0), T(0)};
    V4<T> Q[8];
    for (int i = 0; i < n; ++i) Q[i] = scale4(sub4(P[i + 1], P[i]), T(n));
    for (int k = 1; k < n; ++k)
        for (int i = 0; i < n - k; ++i) Q[i] = mix4(Q[i], Q[i + 1], u);
    return Q[0];
}
// Homogeneous point and partials, BezierPatchOps::BezierPatchEval,
// src/math/bezier_patch.h:172-191.  P is (p+1) x (q+1), index i*(q+1)+j.
template <class T>
static void patch_eval(const V4<T>* P, int p, int q, T u, T v, V4<T>& S, V4<T>& Su, V4<T>& Sv) {
    V4<T> C[8];
    for (int i = 0; i <= p; ++i) C[i] = curve_point(P + i * (q + 1), q, v);
    Su = curve_deriv(C, p, u);
    S = curve_point(C, p, u);
    for (int j = 0; j <= q; ++j) {
        V4<T> col[8];
        for (int i = 0; i <= p; ++i) col[i] = P[i * (q + 1) + j];
        C[j] = curve_point(col, p, u);
    }
    Sv = curve_deriv(C, q, v);
}

// PCG hash (src/math/math_utils.h:12-17) and randf (:70-74).
static inline uint32_t pcg(uint32_t x) {
    x = x * 747796405u + 2891336453u;
    uint32_t w = ((x >> ((x >> 28u) + 4u)) ^ x) * 277803737u;
    return (w >> 22u) ^ w;
}
template <class T> static inline T rand01(uint32_t& s);
template <> inline float rand01<float>(uint32_t& s) { s = pcg(s); return s * 2.3283064e-10f; }
template <> inline double rand01<double>(uint32_t& s) { s = pcg(s); return s * 2.3283064365386963e-10; }

template <class T> struct NewtonResult {
    bool hit;
    V3<T> S, Su, Sv;
    T u, v;
    int evals;
};

// Newton-Raphson on the two ray planes, BezierPatchOps::newtonRhapson,
// src/math/bezier_patch.h:197-266.  The iteration cap is a parameter here
// (the reference fixes it with NEWTON_MAX_ITERATIONS, src/constants.h:38-39).
template <class T>
static NewtonResult<T> newton(const Planes<T>& pl, const V4<T>* P, int p, int q, T u0, T v0, T det_eps,
                              T eps, uint32_t seed, int max_iter) {
    T u = u0, v = v0;
    const T pull = std::is_same<T, float>::value ? T(0.1f) : T(0.1);
    for (int it = 1; it <= max_iter; ++it) {
        V4<T> H, Hu, Hv;
        patch_eval(P, p, q, u, v, H, Hu, Hv);
        const T iw = T(1) / H.w;
        V3<T> S = {H.x * iw, H.y * iw, H.z * iw};
        V3<T> Su = {(Hu.x - S.x * Hu.w) * iw, (Hu.y - S.y * Hu.w) * iw, (Hu.z - S.z * Hu.w) * iw};
        V3<T> Sv = {(Hv.x - S.x * Hv.w) * iw, (Hv.y - S.y * Hv.w) * iw, (Hv.z - S.z * Hv.w) * iw};
        const T r0 = dot3(pl.n1, S) + pl.d1, r1 = dot3(pl.n2, S) + pl.d2;
        const T err = std::fabs(r0) + std::fabs(r1);
        if (err < eps) return {true, S, Su, Sv, u, v, it};
        // Jacobian, column-major as MathTypes::matrix2x2f (bezier_patch.h:236-239)
        const T j0 = dot3(pl.n1, Su), j1 = dot3(pl.n2, Su), j2 = dot3(pl.n1, Sv), j3 = dot3(pl.n2, Sv);
        const T rnd1 = rand01<T>(seed), rnd2 = rand01<T>(seed);
        const T det = j0 * j3 - j2 * j1;  // matrix_ops.h:14-17
        if (std::fabs(det) < det_eps) {
            u = u + pull * ((u0 - u) * rnd1);
            v = v + pull * ((v0 - v) * rnd2);
        } else {  // adjugate / det, then mat * vec (matrix_ops.h:20-32)
            const T i0 = j3 / det, i1 = -j1 / det, i2 = -j2 / det, i3 = j0 / det;
            u = u - (i0 * r0 + i2 * r1);
            v = v - (i1 * r0 + i3 * r1);
        }
        u = std::fmin(std::fmax(u, T(0)), T(1));
        v = std::fmin(std::fmax(v, T(0)), T(1));
    }
    NewtonResult<T> miss{};
    miss.hit = false;
    miss.evals = max_iter;
    return miss;
}

// Ray / bilinear-patch initial guess through the four corners,
// BezierPatchOps::biliniearRay, src/math/bezier_patch.h:272-327.
// Restated as written: the reference forms n = d x pb and then takes n.pb and
// n.d, both identically zero up to rounding, so it returns (0.5, 0.5) unless
// rounding noise makes n.pb positive.  The float instantiation reproduces that
// noise exactly when built without FMA contraction.
template <class T>
static void bilinear_guess(V3<T> q00, V3<T> q10, V3<T> q11, V3<T> q01, V3<T> o, V3<T> d, T& gu, T& gv) {
    const V3<T> e10 = sub3(q10, q00), e11 = sub3(q11, q10), e00 = sub3(q01, q00);
    const V3<T> qn = cross3(e10, sub3(q01, q11));
    q00 = sub3(q00, o);
    q10 = sub3(q10, o);
    const T a = dot3(cross3(q00, d), e00);
    const T c = dot3(qn, d);
    T b = dot3(cross3(q10, d), e11);
    b -= a + c;
    T det = b * b - T(4) * a * c;
    gu = T(0.5); gv = T(0.5);
    if (det < 0) return;
    det = std::sqrt(det);
    T ux[2];
    if (c == 0) { ux[0] = -a / b; ux[1] = -1; }
    else { ux[0] = (-b - std::copysign(det, b)) / 2; ux[1] = a / ux[0]; ux[0] /= c; }
    T best = INFINITY;
    for (int i = 0; i < 2; ++i) {
        if (ux[i] < 0 || ux[i] > 1) continue;
        const T w = T(1) - ux[i];
        const V3<T> pb = {e00.x * w + e11.x * ux[i], e00.y * w + e11.y * ux[i], e00.z * w + e11.z * ux[i]};
        const V3<T> n = cross3(d, pb);
        const T dd = dot3(n, n);
        const T tx = dot3(n, pb);
        const T vx = dot3(n, d);
        if (tx > 0 && 0 <= vx && vx <= dd && tx < best) { gu = ux[i]; gv = vx / dd; best = tx; }
    }
}

}  // namespace orc

using namespace orc;

// ===========================================================================
// extern "C" entry points (plain pointers; all arrays row-major, float32
// unless named *_f64).
extern "C" {

// Number of Bezier pieces along u and v for one surface (segs(), bezier_patch.h:46-53).
int orc_patch_grid(const float* U, const float* V, int n, int m, int p, int q, int* nbU, int* nbV) {
    std::vector<float> bu(n - p + 2), bv(m - q + 2);
    *nbU = breakpoints(U, n + p + 1, p, bu.data());
    *nbV = breakpoints(V, m + q + 1, q, bv.data());
    return 0;
}

// Decompose one NURBS surface into nbU*nbV Bezier patches, as
// BezierPatchOps::getPatch (src/math/bezier_patch.h:86-139): patch (i,j) at
// i*nbV+j, each (p+1)*(q+1) weighted-homogeneous points, index r*(q+1)+c.
// ranges receives (u0,u1,v0,v1) per patch.  f64 != 0 runs the same algorithm
// in double (the FP64 oracle's patches) and writes doubles to cp_out_f64.
int orc_decompose(const float* cp, const float* U, const float* V, int n, int m, int p, int q,
                  float* cp_out, double* cp_out_f64, float* ranges) {
    int nbU, nbV;
    std::vector<float> bu(n - p + 2), bv(m - q + 2);
    nbU = breakpoints(U, n + p + 1, p, bu.data());
    nbV = breakpoints(V, m + q + 1, q, bv.data());
    const int strip = (p + 1) * (m + 1), piece = (p + 1) * (q + 1);
    auto run = [&](auto zero) {
        using T = decltype(zero);
        std::vector<V4<T>> P((size_t)(n + 1) * (m + 1));
        for (size_t i = 0; i < P.size(); ++i) P[i] = {T(cp[4 * i]), T(cp[4 * i + 1]), T(cp[4 * i + 2]), T(cp[4 * i + 3])};
        std::vector<V4<T>> strips((size_t)(nbU + 1) * strip), out((size_t)(nbU * nbV + 1) * piece);
        split_bezier<T>(n, p, U, m, q, V, 0, P.data(), strips.data());
        for (int s = 0; s < nbU; ++s)  // the V pass runs per strip with n = p (bezier_patch.h:106-114)
            split_bezier<T>(p, p, U, m, q, V, 1, strips.data() + (size_t)s * strip, out.data() + (size_t)s * nbV * piece);
        return out;
    };
    if (cp_out) {
        auto out = run(0.0f);
        std::memcpy(cp_out, out.data(), sizeof(float) * 4 * (size_t)nbU * nbV * piece);
    }
    if (cp_out_f64) {
        auto out = run(0.0);
        std::memcpy(cp_out_f64, out.data(), sizeof(double) * 4 * (size_t)nbU * nbV * piece);
    }
    if (ranges)
        for (int i = 0; i < nbU; ++i)
            for (int j = 0; j < nbV; ++j) {
                float* r = ranges + 4 * (i * nbV + j);
                r[0] = bu[i]; r[1] = bu[i + 1]; r[2] = bv[j]; r[3] = bv[j + 1];
            }
    return nbU * nbV;
}

// Patch boxes (6 floats each) for patches given by cp offsets (in points) and degrees.
void orc_patch_boxes(const float* cp, const int* cp_off, const int* deg, int N, float* boxes) {
    for (int k = 0; k < N; ++k)
        patch_box(cp + 4 * (size_t)cp_off[k], (deg[2 * k] + 1) * (deg[2 * k + 1] + 1), boxes + 6 * k);
}

// Exhaustive-SAH binary BVH over boxes.  Outputs up to 2N-1 nodes; returns the
// node count used.  order[k] = original index of the primitive in BVH slot k
// (the reference reorders its patch array the same way, bvh.h:167-175).
int orc_build_bvh(const float* boxes, int N, float* node_box, uint32_t* left_first, uint32_t* prim_count,
                  int32_t* order) {
    std::vector<Box> prim(N);
    for (int i = 0; i < N; ++i)
        for (int k = 0; k < 3; ++k) { prim[i].lo[k] = boxes[6 * i + k]; prim[i].hi[k] = boxes[6 * i + 3 + k]; }
    std::vector<Box> nb(2 * (size_t)N);
    SahBuilder B{prim.data(), std::vector<uint32_t>(N), nb.data(), left_first, prim_count, 1};
    Box root = box_empty();
    for (int i = 0; i < N; ++i) { B.order[i] = i; root = box_join(root, prim[i]); }
    nb[0] = root;
    left_first[0] = 0;
    prim_count[0] = N;
    B.split(0);
    for (int i = 0; i < B.used; ++i)
        for (int k = 0; k < 3; ++k) { node_box[6 * i + k] = nb[i].lo[k]; node_box[6 * i + 3 + k] = nb[i].hi[k]; }
    for (int i = 0; i < N; ++i) order[i] = (int32_t)B.order[i];
    return B.used;
}

// 32-bin SAH binary BVH, the O(N log N) builder this project uses for scenes
// in place of the exhaustive one above (whose O(N^2) levels take minutes at
// 10k patches); the closest hit does not depend on the tree.  Restated from
// its definition (one float rounding per operation): per node the centroid
// bounds, 32 bins along each axis of positive extent, the cost
// nL*halfArea(L) + nR*halfArea(R) at every bin boundary with the first
// minimum in (axis, boundary) order, a stable partition, children numbered as
// a depth-first stack allocates them, leaves where no split separates the
// patches or count <= max_leaf.  Returns the node count used.
int orc_build_bvh_binned(const float* boxes, int N, int max_leaf, float* node_box, uint32_t* lf, uint32_t* cnt,
                         int32_t* order) {
    if (N <= 0) return 0;
    std::vector<Box> prim(N);
    std::vector<float> cen(3 * (size_t)N);
    Box root = box_empty();
    for (int i = 0; i < N; ++i) {
        for (int k = 0; k < 3; ++k) {
            prim[i].lo[k] = boxes[6 * i + k];
            prim[i].hi[k] = boxes[6 * i + 3 + k];
            cen[3 * (size_t)i + k] = 0.5f * (prim[i].lo[k] + prim[i].hi[k]);
        }
        root = box_join(root, prim[i]);
        order[i] = i;
    }
    auto put = [&](int node, const Box& b) {
        for (int k = 0; k < 3; ++k) { node_box[6 * node + k] = b.lo[k]; node_box[6 * node + 3 + k] = b.hi[k]; }
    };
    auto bin_of = [](float c, float l, float s) {
        const float v = (c - l) * s;
        return v >= 0.f ? (v < 32.f ? (int)v : 31) : 0;
    };
    put(0, root);
    lf[0] = 0;
    cnt[0] = (uint32_t)N;
    int used = 1;
    std::vector<int> todo{0};
    std::vector<int32_t> tmp;
    while (!todo.empty()) {
        const int node = todo.back();
        todo.pop_back();
        const uint32_t first = lf[node], count = cnt[node];
        if ((int)count <= max_leaf) continue;
        float clo[3] = {INFINITY, INFINITY, INFINITY}, chi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (uint32_t i = first; i < first + count; ++i)
            for (int k = 0; k < 3; ++k) {
                clo[k] = fminf(clo[k], cen[3 * (size_t)order[i] + k]);
                chi[k] = fmaxf(chi[k], cen[3 * (size_t)order[i] + k]);
            }
        float scale[3];
        Box bins[3][32];
        int bc[3][32] = {};
        float best_c = INFINITY;
        int best_a = -1, best_s = 0;
        for (int a = 0; a < 3; ++a) {
            const float ext = chi[a] - clo[a];
            scale[a] = ext > 0.f ? 32.f / ext : 0.f;
            if (!(ext > 0.f)) continue;
            for (int b = 0; b < 32; ++b) bins[a][b] = box_empty();
            for (uint32_t i = first; i < first + count; ++i) {
                const int b = bin_of(cen[3 * (size_t)order[i] + a], clo[a], scale[a]);
                ++bc[a][b];
                bins[a][b] = box_join(bins[a][b], prim[order[i]]);
            }
            float ra[32];
            int rc[32];
            Box r = box_empty();
            int n = 0;
            for (int k = 31; k >= 1; --k) {
                r = box_join(r, bins[a][k]);
                n += bc[a][k];
                ra[k] = box_half_area(r);
                rc[k] = n;
            }
            Box l = box_empty();
            n = 0;
            for (int k = 0; k < 31; ++k) {
                l = box_join(l, bins[a][k]);
                n += bc[a][k];
                if (n == 0 || rc[k + 1] == 0) continue;
                const float c = (float)n * box_half_area(l) + (float)rc[k + 1] * ra[k + 1];
                if (c < best_c) { best_c = c; best_a = a; best_s = k + 1; }
            }
        }
        if (best_a < 0) continue;
        tmp.clear();
        uint32_t nl = 0;
        for (uint32_t i = first; i < first + count; ++i)
            if (bin_of(cen[3 * (size_t)order[i] + best_a], clo[best_a], scale[best_a]) < best_s) {
                order[first + nl++] = order[i];
            } else {
                tmp.push_back(order[i]);
            }
        if (nl == 0 || nl == count) {  // restore (stable) and keep the node a leaf
            std::vector<int32_t> all;
            for (uint32_t i = first; i < first + nl; ++i) all.push_back(order[i]);
            all.insert(all.end(), tmp.begin(), tmp.end());
            for (uint32_t i = 0; i < count; ++i) order[first + i] = all[i];
            continue;
        }
        for (size_t i = 0; i < tmp.size(); ++i) order[first + nl + i] = tmp[i];
        const int L = used, R = used + 1;
        used += 2;
        Box bl = box_empty(), br = box_empty();
        for (int b = 0; b < best_s; ++b) bl = box_join(bl, bins[best_a][b]);
        for (int b = best_s; b < 32; ++b) br = box_join(br, bins[best_a][b]);
        lf[L] = first; cnt[L] = nl;
        lf[R] = first + nl; cnt[R] = count - nl;
        put(L, bl);
        put(R, br);
        lf[node] = (uint32_t)L;
        cnt[node] = 0;
        todo.push_back(L);
        todo.push_back(R);
    }
    return used;
}

// Options shared by the intersect entry points.
struct orc_opts {
    int init_mode;        // 0 = patch midpoint (0.5,0.5), 1 = reference bilinear guess
    int max_iter;         // Newton evaluations per (ray, patch)
    float eps;            // residual threshold |r1|+|r2| < eps
    float det_eps;        // singular-Jacobian threshold on |det J|
    float flat_threshold; // flat-skip threshold in pixels; 0 disables
    float cam_k;          // 0.5*H/tan(fov/2), only used by flat-skip
};

}  // extern "C"

// Closest hit per ray by the reference's traversal (calculateIntersect,
// src/gpu/intersect.cu:33-193), on a binary BVH in the reference layout whose
// leaves index patches in BVH order (patch k of the BVH = input patch order[k]).
// T = float reproduces the reference's FP32 path; T = double is the FP64 oracle
// (its control points come from cp_f64).
template <class T>
static void intersect_impl(const V4<T>* cp, const int* cp_off, const int* deg, const float* delta,
                           const float* node_box, const uint32_t* lf, const uint32_t* cnt, const int32_t* order,
                           const float* ox, const float* oy, const float* oz, const float* dx, const float* dy,
                           const float* dz, long R, const orc_opts& op, int32_t* hit_patch, T* t_out, T* u_out,
                           T* v_out, int32_t* evals_out, int32_t* tests_out, T* geo_out,
                           unsigned long long* newton_total, unsigned long long* skip_total) {
    unsigned long long nc_all = 0, sc_all = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : nc_all, sc_all)
    for (long idx = 0; idx < R; ++idx) {
        const V3<T> o = {T(ox[idx]), T(oy[idx]), T(oz[idx])};
        const V3<T> d = {T(dx[idx]), T(dy[idx]), T(dz[idx])};
        const float of[3] = {ox[idx], oy[idx], oz[idx]};
        // Box tests stay in float in both instantiations: the BVH is a float structure.
        const float rd[3] = {1 / dx[idx], 1 / dy[idx], 1 / dz[idx]};
        const Planes<T> pl = ray_planes<T>(o, d);
        int stack[64];
        int sp = 0;
        T t_max = INFINITY;
        int best = -1, best_evals = 0, tests = 0;
        T bu = 0, bv = 0;
        V3<T> bS{}, bSu{}, bSv{};
        unsigned long long nc = 0, sc = 0;
        uint32_t node = 0;
        float t_box = slab(node_box, of, rd);
        bool live = t_box < (float)t_max;
        while (live) {
            if (cnt[node] > 0) {
                t_box = slab(node_box + 6 * node, of, rd);
                for (uint32_t i = 0; i < cnt[node]; ++i) {
                    const int slot = (int)(lf[node] + i);
                    const int k = order[slot];
                    const V4<T>* P = cp + cp_off[k];
                    const int p = deg[2 * k], q = deg[2 * k + 1];
                    ++tests;
                    T gu = T(0.5), gv = T(0.5);
                    if (op.init_mode == 1)  // corners(), bezier_patch.h:37-44
                        bilinear_guess<T>(dehom(P[0]), dehom(P[p * (q + 1)]), dehom(P[p * (q + 1) + q]), dehom(P[q]),
                                          o, d, gu, gv);
                    bool do_newton = true;
                    if (delta && op.flat_threshold > 0 && delta[slot] * op.cam_k / t_box < op.flat_threshold) {
                        // flat-skip, intersect.cu:104-123 with evalPointNormal (bezier_patch.h:330-340)
                        V4<T> H, Hu, Hv;
                        patch_eval(P, p, q, gu, gv, H, Hu, Hv);
                        const T iw = T(1) / H.w;
                        V3<T> S = {H.x * iw, H.y * iw, H.z * iw};
                        V3<T> Su = {(Hu.x - S.x * Hu.w) * iw, (Hu.y - S.y * Hu.w) * iw, (Hu.z - S.z * Hu.w) * iw};
                        V3<T> Sv = {(Hv.x - S.x * Hv.w) * iw, (Hv.y - S.y * Hv.w) * iw, (Hv.z - S.z * Hv.w) * iw};
                        const T res = std::fabs(dot3(pl.n1, S) + pl.d1) + std::fabs(dot3(pl.n2, S) + pl.d2);
                        if (res * op.cam_k / t_box < op.flat_threshold) {
                            ++sc;
                            const T t = dot3(sub3(S, o), d);
                            if (0 < t && t < t_max) {
                                t_max = t; best = k; bu = gu; bv = gv; bS = S; bSu = Su; bSv = Sv; best_evals = 0;
                                do_newton = false;
                            }
                        }
                    }
                    if (do_newton) {
                        ++nc;
                        NewtonResult<T> r = newton<T>(pl, P, p, q, gu, gv, T(op.det_eps), T(op.eps), (uint32_t)idx,
                                                      op.max_iter);
                        if (r.hit) {
                            const T t = (r.S.x - o.x) * d.x + (r.S.y - o.y) * d.y + (r.S.z - o.z) * d.z;
                            if (0 < t && t < t_max) {
                                t_max = t; best = k; bu = r.u; bv = r.v; bS = r.S; bSu = r.Su; bSv = r.Sv;
                                best_evals = r.evals;
                            }
                        }
                    }
                }
                if (sp == 0) break;
                node = (uint32_t)stack[--sp];
            } else {
                const uint32_t L = lf[node], Rn = L + 1;
                const float tl = slab(node_box + 6 * L, of, rd), tr = slab(node_box + 6 * Rn, of, rd);
                const float tn = fminf(tl, tr);
                if (tn >= (float)t_max) {
                    if (sp == 0) break;
                    node = (uint32_t)stack[--sp];
                } else if (tl <= tn) {
                    if (tr < (float)t_max && sp < 64) stack[sp++] = (int)Rn;
                    node = L;
                } else {
                    if (tl < (float)t_max && sp < 64) stack[sp++] = (int)L;
                    node = Rn;
                }
            }
        }
        nc_all += nc;
        sc_all += sc;
        hit_patch[idx] = best;
        if (t_out) t_out[idx] = best >= 0 ? t_max : T(-1);
        if (u_out) u_out[idx] = bu;
        if (v_out) v_out[idx] = bv;
        if (evals_out) evals_out[idx] = best_evals;
        if (tests_out) tests_out[idx] = tests;
        if (geo_out) {
            T* g = geo_out + 9 * idx;
            g[0] = bS.x; g[1] = bS.y; g[2] = bS.z;
            g[3] = bSu.x; g[4] = bSu.y; g[5] = bSu.z;
            g[6] = bSv.x; g[7] = bSv.y; g[8] = bSv.z;
        }
    }
    if (newton_total) *newton_total = nc_all;
    if (skip_total) *skip_total = sc_all;
}

extern "C" {

void orc_intersect_f32(const float* cp, const int* cp_off, const int* deg, const float* delta,
                       const float* node_box, const uint32_t* lf, const uint32_t* cnt, const int32_t* order,
                       const float* ox, const float* oy, const float* oz, const float* dx, const float* dy,
                       const float* dz, long R, const orc_opts* op, int32_t* hit_patch, float* t, float* u, float* v,
                       int32_t* evals, int32_t* tests, float* geo, unsigned long long* newton_total,
                       unsigned long long* skip_total) {
    intersect_impl<float>(reinterpret_cast<const V4<float>*>(cp), cp_off, deg, delta, node_box, lf, cnt, order, ox, oy,
                          oz, dx, dy, dz, R, *op, hit_patch, t, u, v, evals, tests, geo, newton_total, skip_total);
}

void orc_intersect_f64(const double* cp, const int* cp_off, const int* deg, const float* delta,
                       const float* node_box, const uint32_t* lf, const uint32_t* cnt, const int32_t* order,
                       const float* ox, const float* oy, const float* oz, const float* dx, const float* dy,
                       const float* dz, long R, const orc_opts* op, int32_t* hit_patch, double* t, double* u,
                       double* v, int32_t* evals, int32_t* tests, double* geo, unsigned long long* newton_total,
                       unsigned long long* skip_total) {
    intersect_impl<double>(reinterpret_cast<const V4<double>*>(cp), cp_off, deg, delta, node_box, lf, cnt, order, ox,
                           oy, oz, dx, dy, dz, R, *op, hit_patch, t, u, v, evals, tests, geo, newton_total,
                           skip_total);
}

// "True closest hit" diagnostic (FP64, multi-start).  Newton from the patch
// midpoint (the method) finds at most one root of each patch it tests, and the
// root it finds depends on the basin the start lies in; when the engine and
// the FP64 oracle disagree, this tells "another root of the same surface" and
// "a root the single start missed" apart from a wrong answer.  For every ray
// and every patch whose box (widened by 1e-4 of its extent) the ray crosses,
// plain Newton in double (no random pull: a singular step abandons the start)
// runs from a grid x grid lattice of starts ((i + 1/2) / grid) and from
// (1/2, 1/2), up to max_iter steps, converged when |r1| + |r2| < eps; the roots
// with t > 0 are collected, coincident ones (|du| + |dv| < 1e-7 on one patch)
// counted once.  Output per ray: the nearest root (patch in input order, -1
// if none; t, u, v) and the number of distinct roots.  With only_patch set,
// polish mode: one start (u0[i], v0[i]) on patch only_patch[i] (< 0: skipped),
// no box test; patch_out[i] = only_patch[i] if it converged, else -1.
static bool newton_polish(const Planes<double>& pl, const V4<double>* P, int p, int q, double& u, double& v,
                          int max_iter, double eps, V3<double>& S_out) {
    for (int it = 0; it < max_iter; ++it) {
        V4<double> H, Hu, Hv;
        patch_eval(P, p, q, u, v, H, Hu, Hv);
        const double iw = 1.0 / H.w;
        const V3<double> S = {H.x * iw, H.y * iw, H.z * iw};
        const V3<double> Su = {(Hu.x - S.x * Hu.w) * iw, (Hu.y - S.y * Hu.w) * iw, (Hu.z - S.z * Hu.w) * iw};
        const V3<double> Sv = {(Hv.x - S.x * Hv.w) * iw, (Hv.y - S.y * Hv.w) * iw, (Hv.z - S.z * Hv.w) * iw};
        const double r0 = dot3(pl.n1, S) + pl.d1, r1 = dot3(pl.n2, S) + pl.d2;
        if (std::fabs(r0) + std::fabs(r1) < eps) {
            S_out = S;
            return true;
        }
        const double j0 = dot3(pl.n1, Su), j1 = dot3(pl.n2, Su), j2 = dot3(pl.n1, Sv), j3 = dot3(pl.n2, Sv);
        const double det = j0 * j3 - j2 * j1;
        if (det == 0.0 || !std::isfinite(det)) return false;
        u = std::fmin(std::fmax(u - (j3 * r0 - j2 * r1) / det, 0.0), 1.0);
        v = std::fmin(std::fmax(v - (j0 * r1 - j1 * r0) / det, 0.0), 1.0);
    }
    return false;
}

void orc_roots_f64(const double* cp, const int* cp_off, const int* deg, const float* boxes, int N, const float* ox,
                   const float* oy, const float* oz, const float* dx, const float* dy, const float* dz, long R,
                   int grid, int max_iter, double eps, const int32_t* only_patch, const double* u0,
                   const double* v0, int32_t* patch_out, double* t_out, double* u_out, double* v_out,
                   int32_t* n_roots_out) {
#pragma omp parallel for schedule(dynamic, 16)
    for (long i = 0; i < R; ++i) {
        const V3<double> o = {ox[i], oy[i], oz[i]}, d = {dx[i], dy[i], dz[i]};
        const Planes<double> pl = ray_planes<double>(o, d);
        patch_out[i] = -1;
        t_out[i] = -1.0;
        u_out[i] = v_out[i] = 0.0;
        if (n_roots_out) n_roots_out[i] = 0;
        auto t_of = [&](const V3<double>& S) { return (S.x - o.x) * d.x + (S.y - o.y) * d.y + (S.z - o.z) * d.z; };
        if (only_patch) {
            const int k = only_patch[i];
            if (k < 0) continue;
            double u = u0[i], v = v0[i];
            V3<double> S;
            if (newton_polish(pl, reinterpret_cast<const V4<double>*>(cp) + cp_off[k], deg[2 * k], deg[2 * k + 1], u,
                              v, max_iter, eps, S)) {
                patch_out[i] = k;
                t_out[i] = t_of(S);
                u_out[i] = u;
                v_out[i] = v;
            }
            continue;
        }
        const float of[3] = {ox[i], oy[i], oz[i]};
        const float rd[3] = {1 / dx[i], 1 / dy[i], 1 / dz[i]};
        double best = INFINITY;
        int n_roots = 0;
        std::vector<double> ru, rv;
        for (int k = 0; k < N; ++k) {
            float b[6];
            for (int a = 0; a < 3; ++a) {
                const float w = 1e-4f * (boxes[6 * k + 3 + a] - boxes[6 * k + a]) + 1e-6f;
                b[a] = boxes[6 * k + a] - w;
                b[3 + a] = boxes[6 * k + 3 + a] + w;
            }
            if (!(slab(b, of, rd) < INFINITY)) continue;
            const V4<double>* P = reinterpret_cast<const V4<double>*>(cp) + cp_off[k];
            const int p = deg[2 * k], q = deg[2 * k + 1];
            ru.clear();
            rv.clear();
            for (int s = 0; s <= grid * grid; ++s) {
                double u = s == grid * grid ? 0.5 : (s / grid + 0.5) / grid;
                double v = s == grid * grid ? 0.5 : (s % grid + 0.5) / grid;
                V3<double> S;
                if (!newton_polish(pl, P, p, q, u, v, max_iter, eps, S)) continue;
                const double t = t_of(S);
                if (!(t > 0)) continue;
                bool seen = false;
                for (size_t r = 0; r < ru.size() && !seen; ++r) seen = std::fabs(ru[r] - u) + std::fabs(rv[r] - v) < 1e-7;
                if (seen) continue;
                ru.push_back(u);
                rv.push_back(v);
                ++n_roots;
                if (t < best) {
                    best = t;
                    patch_out[i] = k;
                    t_out[i] = t;
                    u_out[i] = u;
                    v_out[i] = v;
                }
            }
        }
        if (n_roots_out) n_roots_out[i] = n_roots;
    }
}

// Single (ray, patch) Newton solve, for unit tests of the per-patch step.
int orc_newton_f32(const float* cp, int p, int q, const float* o, const float* d, float u0, float v0, float det_eps,
                   float eps, uint32_t seed, int max_iter, float* out /* u, v, S(3), Su(3), Sv(3) */) {
    Planes<float> pl = ray_planes<float>({o[0], o[1], o[2]}, {d[0], d[1], d[2]});
    auto r = newton<float>(pl, reinterpret_cast<const V4<float>*>(cp), p, q, u0, v0, det_eps, eps, seed, max_iter);
    out[0] = r.u; out[1] = r.v;
    out[2] = r.S.x; out[3] = r.S.y; out[4] = r.S.z;
    out[5] = r.Su.x; out[6] = r.Su.y; out[7] = r.Su.z;
    out[8] = r.Sv.x; out[9] = r.Sv.y; out[10] = r.Sv.z;
    return r.hit ? r.evals : -r.evals;
}

// Homogeneous point and partials of one patch (float or double).
void orc_patch_eval_f64(const double* cp, int p, int q, double u, double v, double* out12) {
    V4<double> S, Su, Sv;
    patch_eval<double>(reinterpret_cast<const V4<double>*>(cp), p, q, u, v, S, Su, Sv);
    double vals[12] = {S.x, S.y, S.z, S.w, Su.x, Su.y, Su.z, Su.w, Sv.x, Sv.y, Sv.z, Sv.w};
    std::memcpy(out12, vals, sizeof(vals));
}

// Ray planes (float), for unit tests.
void orc_ray_planes_f32(const float* o, const float* d, float* out8) {
    Planes<float> pl = ray_planes<float>({o[0], o[1], o[2]}, {d[0], d[1], d[2]});
    float vals[8] = {pl.n1.x, pl.n1.y, pl.n1.z, pl.n2.x, pl.n2.y, pl.n2.z, pl.d1, pl.d2};
    std::memcpy(out8, vals, sizeof(vals));
}

// Rational surface point by Algorithms A2.1/A2.2/A4.3 in double
// (NurbsOps::findSpan/basisFuncEval/surfacePoint, src/math/nurbs.h:34-92);
// used to check that decomposition preserves the surface.
static int span_of(int n, int p, double u, const double* U) {
    if (u >= U[n + 1]) return n;
    int lo = p, hi = n + 1, mid = (lo + hi) / 2;
    while (u < U[mid] || u >= U[mid + 1]) {
        if (u < U[mid]) hi = mid; else lo = mid;
        mid = (lo + hi) / 2;
    }
    return mid;
}
static void basis(int i, double u, int p, const double* U, double* N) {
    double left[9], right[9];
    N[0] = 1.0;
    for (int j = 1; j <= p; ++j) {
        left[j] = u - U[i + 1 - j];
        right[j] = U[i + j] - u;
        double saved = 0.0;
        for (int r = 0; r < j; ++r) {
            double tmp = N[r] / (right[r + 1] + left[j - r]);
            N[r] = saved + right[r + 1] * tmp;
            saved = left[j - r] * tmp;
        }
        N[j] = saved;
    }
}
void orc_surface_point_f64(const float* cp, const float* Uf, const float* Vf, int n, int m, int p, int q, double u,
                           double v, double* out3) {
    std::vector<double> U(Uf, Uf + n + p + 2), V(Vf, Vf + m + q + 2);
    double Nu[9], Nv[9];
    int su = span_of(n, p, u, U.data()), sv = span_of(m, q, v, V.data());
    basis(su, u, p, U.data(), Nu);
    basis(sv, v, q, V.data(), Nv);
    double acc[4] = {0, 0, 0, 0};
    for (int k = 0; k <= p; ++k)
        for (int l = 0; l <= q; ++l) {
            const float* c = cp + 4 * ((size_t)(su - p + k) * (m + 1) + (sv - q + l));
            for (int e = 0; e < 4; ++e) acc[e] += Nu[k] * Nv[l] * (double)c[e];
        }
    out3[0] = acc[0] / acc[3]; out3[1] = acc[1] / acc[3]; out3[2] = acc[2] / acc[3];
}

// Pinhole camera rays, the reference's perspective camera (Transform::lookAt,
// src/math/transform.h:46-60; CameraOps::init_camera/getPerspectiveCamera/
// calculateRay<perspective_projection>, src/core/camera.h:63-174) reduced to its
// closed form and evaluated in double:
//   screen window [-a,a]x[-1,1] (a = W/H >= 1, else [-1,1]x[-1/a,1/a]),
//   camera-space direction normalize(sx*tan(fov/2), sy*tan(fov/2), 1),
//   world direction = [right | up' | forward] * d_cam, origin = eye.
// spp > 1 jitters the sample inside the pixel with a seeded PCG hash; spp == 1
// uses the pixel centre (+0.5) as the reference does.  Ray index =
// (y*W + x)*spp + s.
void orc_camera_rays(const float* eye, const float* look, const float* up, float fov_deg, int W, int H, int spp,
                     uint32_t seed, float* ox, float* oy, float* oz, float* dx, float* dy, float* dz) {
    auto norm = [](V3<double> a) { double l = std::sqrt(dot3(a, a)); return scale3(a, 1.0 / l); };
    V3<double> E = {eye[0], eye[1], eye[2]}, L = {look[0], look[1], look[2]}, Up = {up[0], up[1], up[2]};
    V3<double> fwd = norm(sub3(L, E));
    V3<double> right = norm(cross3(Up, fwd));
    V3<double> nup = cross3(fwd, right);
    const double aspect = double(W) / double(H);
    double x0, x1, y0, y1;
    if (aspect > 1.0) { x0 = -aspect; x1 = aspect; y0 = -1; y1 = 1; }
    else { x0 = -1; x1 = 1; y0 = -1.0 / aspect; y1 = 1.0 / aspect; }
    const double th = std::tan(double(fov_deg) * (3.14159265358979323846 / 180.0) / 2.0);
#pragma omp parallel for schedule(static)
    for (long pix = 0; pix < (long)W * H; ++pix) {
        const int px = (int)(pix % W), py = (int)(pix / W);
        for (int s = 0; s < spp; ++s) {
            const long r = pix * spp + s;
            double jx = 0.5, jy = 0.5;
            if (spp > 1) {
                uint32_t h = pcg(seed ^ pcg((uint32_t)r));
                jx = (double)(h >> 8) * (1.0 / 16777216.0);
                h = pcg(h);
                jy = (double)(h >> 8) * (1.0 / 16777216.0);
            }
            const double sx = x0 + (px + jx) * (x1 - x0) / W;
            const double sy = y1 - (py + jy) * (y1 - y0) / H;
            V3<double> dc = norm(V3<double>{sx * th, sy * th, 1.0});
            V3<double> dw = {right.x * dc.x + nup.x * dc.y + fwd.x * dc.z, right.y * dc.x + nup.y * dc.y + fwd.y * dc.z,
                             right.z * dc.x + nup.z * dc.y + fwd.z * dc.z};
            ox[r] = (float)E.x; oy[r] = (float)E.y; oz[r] = (float)E.z;
            dx[r] = (float)dw.x; dy[r] = (float)dw.y; dz[r] = (float)dw.z;
        }
    }
}

// Flatness of a patch: largest distance between a control point and the
// bilinear interpolation of the four corners at its Greville-like node
// (patchDelta, src/core/main.cpp:18-43 and src/core/benchmark.cpp:34-48).
void orc_patch_delta(const float* cp, const int* cp_off, const int* deg, int N, float* out) {
    for (int k = 0; k < N; ++k) {
        const float* P = cp + 4 * (size_t)cp_off[k];
        const int p = deg[2 * k], q = deg[2 * k + 1], row = q + 1;
        auto dh = [&](int i) { const float* c = P + 4 * i; float iw = 1.0f / c[3]; return V3<float>{c[0] * iw, c[1] * iw, c[2] * iw}; };
        V3<float> c00 = dh(0), c10 = dh(p * row), c01 = dh(q), c11 = dh(p * row + q);
        float dmax = 0;
        for (int i = 0; i <= p; ++i)
            for (int j = 0; j <= q; ++j) {
                float u = (float)i / p, v = (float)j / q;
                float a = (1 - u) * (1 - v), b = u * (1 - v), c = (1 - u) * v, e = u * v;
                V3<float> B = {a * c00.x + b * c10.x + c * c01.x + e * c11.x, a * c00.y + b * c10.y + c * c01.y + e * c11.y,
                               a * c00.z + b * c10.z + c * c01.z + e * c11.z};
                V3<float> Pij = dh(i * row + j);
                float ddx = Pij.x - B.x, ddy = Pij.y - B.y, ddz = Pij.z - B.z;
                dmax = fmaxf(dmax, sqrtf(ddx * ddx + ddy * ddy + ddz * ddz));
            }
        out[k] = dmax;
    }
}

}  // extern "C"
