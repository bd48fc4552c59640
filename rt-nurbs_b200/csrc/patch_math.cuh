// patch_math.cuh -- per-(ray, patch) device math of the intersection path.
//
// Patches live on the device in patch-local coordinates: every patch has a
// centre C (double) and its control points are stored as
// (w*(x-Cx), w*(y-Cy), w*(z-Cz), w) in FP32, one block per patch of two
// halves, XY = X0 Y0 X1 Y1 ... and ZW = Z0 W0 Z1 W1 ... (np = (p+1)(q+1)
// rounded up to 4 points per coordinate, 16-byte aligned): a 16-byte load
// brings two points' (x, y) or (z, w) pairs, the operand pairs of the paired
// FP32 instructions that evaluate two coordinates at once.
// The ray's two planes n_k.x + d_k = 0 (MathUtils::getRayPlanes,
// src/math/math_utils.h:33-54) become n_k.S_loc + e_k with e_k = -n_k.(O - C)
// computed in FP64 once per (ray, patch); |e_k| is the distance from the ray to
// the patch centre, so the FP32 residual keeps its precision however far the
// ray origin is from the patch.  The method is the reference's
// (BezierPatchOps::newtonRhapson, src/math/bezier_patch.h:197-266); only the
// coordinate origin and the evaluation scheme differ.
#pragma once

#include <cstdint>

namespace nrt {
namespace dev {

constexpr int kMaxDeg = 7;

__host__ __device__ constexpr int padded_points(int p, int q) { return (((p + 1) * (q + 1)) + 3) & ~3; }

// Offsets (floats) of point k's coordinates in a block of np padded points:
// coordinate a = 0..3 (x, y, z, w) of point k is at block_at(np, k, a).
__host__ __device__ constexpr int block_at(int np, int k, int a) { return (a >> 1) * 2 * np + 2 * k + (a & 1); }

__device__ __forceinline__ float fmx(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fmx(double a, double b, double c) { return ::fma(a, b, c); }

// Packed patch header: x = first float of the SoA block, y = p | q<<4 |
// flags<<8, z = global patch id, w = surface id.
// kFlagWideWeights: the weights span more than kWideWeightRatio (max / min),
// where the FP32 residual's rounding floor approaches the stop rule's eps and
// the FP64 decisions of newton_step apply.
enum : int { kFlagPositiveWeights = 1, kFlagWideWeights = 2 };
constexpr double kWideWeightRatio = 64.0;

struct RayFrame {
    float ox, oy, oz, dx, dy, dz;
    float n1x, n1y, n1z, n2x, n2y, n2z;
};

// Per (ray, patch) offsets, FP32 for the iteration and FP64 for the final step.
struct PatchRay {
    float e1, e2, tc;
    double e1d, e2d, tcd;
    double ocx, ocy, ocz;  // ray origin minus patch centre, in double (the FP64 final step)
};

struct NewtonOpts {
    int max_iter;
    float eps;
    float det_eps;
    float cond_fp64;
    int fp64_final;
    int fp64_band;   // 1: convergence near eps is decided in FP64 (newton_tail_fp64)
};

// The FP64 decision band of the FP64 final-step mode (op.fp64_band, set per
// patch for patches flagged kFlagWideWeights): an FP32 residual below
// kBandLo * eps is accepted as converged, and one in [kBandLo * eps,
// kBandHi * eps) hands the solve to FP64, which continues the same iteration
// from there with the evaluations left (on nets with extreme weights the FP32
// residual has a rounding floor near eps and would stall in this band).
constexpr float kBandLo = 0.125f, kBandHi = 16.f;

struct NewtonOut {
    int evals;       // > 0 converged after this many evaluations; < 0 not converged
    float u, v;
    float t;         // along the ray, in units of |d|
    float sx, sy, sz, ux, uy, uz, vx, vy, vz;  // S (local), dS/du, dS/dv
    int fp64_solves;
    int fp64_final;
    int flat;        // 1: accepted by the flat-skip test at the initial guess (evals 0)
    int done;        // FP32 evaluations actually run (the fixed-point exit ends some solves early)
};

// PCG hash (src/math/math_utils.h:12-17).
__device__ __forceinline__ uint32_t pcg_hash(uint32_t x) {
    x = x * 747796405u + 2891336453u;
    const uint32_t w = ((x >> ((x >> 28u) + 4u)) ^ x) * 277803737u;
    return (w >> 22u) ^ w;
}

// The two planes containing the ray, getRayPlanes (math_utils.h:33-54) with
// IEEE square root and division.
__device__ __forceinline__ void ray_planes(RayFrame& r) {
    const float ax = fabsf(r.dx), ay = fabsf(r.dy), az = fabsf(r.dz);
    const bool xdom = (ax > ay) && (ax > az);
    const float bx = xdom ? r.dx : r.dy, by = xdom ? r.dy : r.dz;
    const float rl = __frcp_rn(__fsqrt_rn(bx * bx + by * by));
    if (xdom) { r.n1x = r.dy * rl; r.n1y = -r.dx * rl; r.n1z = 0.f; }
    else { r.n1x = 0.f; r.n1y = r.dz * rl; r.n1z = -r.dy * rl; }
    const float il = __frcp_rn(__fsqrt_rn(r.dx * r.dx + r.dy * r.dy + r.dz * r.dz));
    const float ux = r.dx * il, uy = r.dy * il, uz = r.dz * il;
    r.n2x = r.n1y * uz - r.n1z * uy;
    r.n2y = r.n1z * ux - r.n1x * uz;
    r.n2z = r.n1x * uy - r.n1y * ux;
}

__device__ __forceinline__ PatchRay patch_ray(const RayFrame& r, double cx, double cy, double cz) {
    const double ox = (double)r.ox - cx, oy = (double)r.oy - cy, oz = (double)r.oz - cz;
    PatchRay pr;
    pr.e1d = -((double)r.n1x * ox + (double)r.n1y * oy + (double)r.n1z * oz);
    pr.e2d = -((double)r.n2x * ox + (double)r.n2y * oy + (double)r.n2z * oz);
    pr.tcd = -((double)r.dx * ox + (double)r.dy * oy + (double)r.dz * oz);
    pr.ocx = ox;
    pr.ocy = oy;
    pr.ocz = oz;
    pr.e1 = (float)pr.e1d;
    pr.e2 = (float)pr.e2d;
    pr.tc = (float)pr.tcd;
    return pr;
}

// Bernstein values of degree N at t, B[i] = C(N,i) t^i (1-t)^(N-i), and their
// derivatives dB[i] = N (B^{N-1}[i-1] - B^{N-1}[i]), from the degree N-1
// values built by the triangle recursion b_i <- (1-t) b_i + t b_{i-1}.
template <int N, class T>
__device__ __forceinline__ void bernstein(T t, T (&B)[N + 1], T (&dB)[N + 1]) {
    const T s = T(1) - t;
    T b[N];
    b[0] = T(1);
#pragma unroll
    for (int k = 1; k < N; ++k) {  // degree k from degree k-1, in place from the top
        b[k] = t * b[k - 1];
#pragma unroll
        for (int i = k - 1; i >= 1; --i) b[i] = fmx(s, b[i], t * b[i - 1]);
        b[0] = s * b[0];
    }
    B[0] = s * b[0];
    B[N] = t * b[N - 1];
    dB[0] = -T(N) * b[0];
    dB[N] = T(N) * b[N - 1];
#pragma unroll
    for (int i = 1; i < N; ++i) {
        B[i] = fmx(s, b[i], t * b[i - 1]);
        dB[i] = T(N) * (b[i - 1] - b[i]);
    }
}

// Tensor-product rational Bezier evaluation as a Bernstein sum: each row i
// of the net is summed along v with the basis values and their derivatives
// (the row point and its v-derivative), then the rows are summed along u.  H,
// dH/du, dH/dv of one coordinate cost 2(p+1)(q+1) + 3(p+1) multiply-adds,
// with the basis values computed once per (u, v) for all four coordinates;
// the reference's BezierPatchEval (src/math/bezier_patch.h:172-191) runs two
// full de Casteljau passes instead.
//
// The four homogeneous coordinates are evaluated as two pairs, (x, y) and
// (z, w), with the paired FP32 instructions of sm_100 (__fmul2_rn,
// __ffma2_rn: one instruction, two round-to-nearest operations, each lane's
// result that of the scalar __fmul_rn / __fmaf_rn): every multiply-add of the
// sum serves two coordinates, and the block stores each point's pairs as
// adjacent floats, so the operand pairs come straight from 16-byte loads.
// Lane by lane the operations and their order are the scalar sum's.
template <int P, int Q>
__device__ __forceinline__ void eval_pair(const float2 (&c)[(P + 1) * (Q + 1)], const float (&Bu)[P + 1],
                                          const float (&dBu)[P + 1], const float2 (&bv)[Q + 1],
                                          const float2 (&dbv)[Q + 1], float2& h, float2& hu, float2& hv) {
#pragma unroll
    for (int i = 0; i <= P; ++i) {
        float2 r = __fmul2_rn(bv[0], c[i * (Q + 1)]), d = __fmul2_rn(dbv[0], c[i * (Q + 1)]);
#pragma unroll
        for (int j = 1; j <= Q; ++j) {
            r = __ffma2_rn(bv[j], c[i * (Q + 1) + j], r);
            d = __ffma2_rn(dbv[j], c[i * (Q + 1) + j], d);
        }
        const float2 bu = make_float2(Bu[i], Bu[i]), dbu = make_float2(dBu[i], dBu[i]);
        if (i == 0) {
            h = __fmul2_rn(bu, r);
            hu = __fmul2_rn(dbu, r);
            hv = __fmul2_rn(bu, d);
        } else {
            h = __ffma2_rn(bu, r, h);
            hu = __ffma2_rn(dbu, r, hu);
            hv = __ffma2_rn(bu, d, hv);
        }
    }
}

// Load one half of a patch block (the (x, y) or the (z, w) pairs of all
// points) with 16-byte loads, two points per load.
template <int P, int Q>
__device__ __forceinline__ void load_pairs(const float* __restrict__ src, float2 (&c)[(P + 1) * (Q + 1)]) {
    constexpr int N = (P + 1) * (Q + 1);
    constexpr int NP = padded_points(P, Q);
    const float4* s4 = reinterpret_cast<const float4*>(src);
#pragma unroll
    for (int k = 0; k < NP / 2; ++k) {
        const float4 f = __ldg(s4 + k);
        if (2 * k + 0 < N) c[2 * k + 0] = make_float2(f.x, f.y);
        if (2 * k + 1 < N) c[2 * k + 1] = make_float2(f.z, f.w);
    }
}

// H, dH/du, dH/dv of the four homogeneous coordinates at (u, v), FP32.
template <int P, int Q>
__device__ __forceinline__ void eval_patch(const float* __restrict__ blk, float u, float v, float (&H)[4],
                                           float (&Hu)[4], float (&Hv)[4]) {
    constexpr int NP = padded_points(P, Q);
    float Bu[P + 1], dBu[P + 1], Bv[Q + 1], dBv[Q + 1];
    bernstein<P, float>(u, Bu, dBu);
    bernstein<Q, float>(v, Bv, dBv);
    float2 bv[Q + 1], dbv[Q + 1];
#pragma unroll
    for (int j = 0; j <= Q; ++j) {
        bv[j] = make_float2(Bv[j], Bv[j]);
        dbv[j] = make_float2(dBv[j], dBv[j]);
    }
#pragma unroll
    for (int a = 0; a < 2; ++a) {  // (x, y), then (z, w)
        float2 c[(P + 1) * (Q + 1)];
        load_pairs<P, Q>(blk + a * 2 * NP, c);
        float2 h, hu, hv;
        eval_pair<P, Q>(c, Bu, dBu, bv, dbv, h, hu, hv);
        H[2 * a] = h.x; H[2 * a + 1] = h.y;
        Hu[2 * a] = hu.x; Hu[2 * a + 1] = hu.y;
        Hv[2 * a] = hv.x; Hv[2 * a + 1] = hv.y;
    }
}

// FP64 evaluation that streams one row at a time from memory, so that high
// degrees do not hold a whole coordinate array in (double) registers.
template <int P, int Q>
__device__ __forceinline__ void eval_patch_fp64(const float* __restrict__ blk, double u, double v, double (&H)[4],
                                                double (&Hu)[4], double (&Hv)[4]) {
    constexpr int NP = padded_points(P, Q);
#pragma unroll 1
    for (int a = 0; a < 4; ++a) {
        const float* __restrict__ src = blk + block_at(NP, 0, a);  // coordinate a of point k at src[2 k]
        double pt[P + 1], dv[P + 1];
#pragma unroll
        for (int i = 0; i <= P; ++i) {
            double r[Q + 1];
#pragma unroll
            for (int j = 0; j <= Q; ++j) r[j] = (double)__ldg(src + 2 * (i * (Q + 1) + j));
#pragma unroll
            for (int k = 1; k < Q; ++k)
#pragma unroll
                for (int j = 0; j <= Q - k; ++j) r[j] = fmx(v, r[j + 1] - r[j], r[j]);
            const double dl = r[1] - r[0];
            pt[i] = fmx(v, dl, r[0]);
            dv[i] = double(Q) * dl;
        }
#pragma unroll
        for (int k = 1; k < P; ++k)
#pragma unroll
            for (int i = 0; i <= P - k; ++i) pt[i] = fmx(u, pt[i + 1] - pt[i], pt[i]);
#pragma unroll
        for (int k = 1; k <= P; ++k)
#pragma unroll
            for (int i = 0; i <= P - k; ++i) dv[i] = fmx(u, dv[i + 1] - dv[i], dv[i]);
        const double dl = pt[1] - pt[0];
        H[a] = fmx(u, dl, pt[0]);
        Hu[a] = double(P) * dl;
        Hv[a] = dv[0];
    }
}

// Ray-space hull test.  For w > 0 the surface point S(u,v), u,v in [0,1], is
// a convex combination of the dehomogenised control points, so the plane
// residual n.S + e is bounded by the control points' residuals.  If every
// control point lies beyond +lim (or below -lim) for either plane, no
// evaluation can meet |r1| + |r2| < eps and Newton's outcome is "no hit":
// the test can be skipped without changing the result.  lim = eps plus a
// rounding margin scaled by the patch radius.
template <int P, int Q>
__device__ __forceinline__ bool hull_misses(const float* __restrict__ blk, const RayFrame& r, const PatchRay& pr,
                                            float lim) {
    constexpr int N = (P + 1) * (Q + 1);
    constexpr int NP = padded_points(P, Q);
    const float4* XY = reinterpret_cast<const float4*>(blk);
    const float4* ZW = reinterpret_cast<const float4*>(blk + 2 * NP);
    bool pos1 = true, neg1 = true, pos2 = true, neg2 = true;
#pragma unroll
    for (int k = 0; k < NP / 2; ++k) {  // two points per pair of loads
        const float4 xy = __ldg(XY + k), zw = __ldg(ZW + k);
        const float xs[2] = {xy.x, xy.z}, ys[2] = {xy.y, xy.w};
        const float zs[2] = {zw.x, zw.z}, ws[2] = {zw.y, zw.w};
#pragma unroll
        for (int l = 0; l < 2; ++l) {
            if (2 * k + l >= N) break;
            const float a = fmaf(r.n1x, xs[l], fmaf(r.n1y, ys[l], fmaf(r.n1z, zs[l], pr.e1 * ws[l])));
            const float b = fmaf(r.n2x, xs[l], fmaf(r.n2y, ys[l], fmaf(r.n2z, zs[l], pr.e2 * ws[l])));
            const float m = lim * ws[l];
            pos1 &= a > m;
            neg1 &= a < -m;
            pos2 &= b > m;
            neg2 &= b < -m;
        }
    }
    return pos1 | neg1 | pos2 | neg2;
}

// Subdivided hull test.  The patch's plane residuals n_k.S + e_k are rational
// Bezier functions whose homogeneous coefficients are a = n1.P + e1*w and
// b = n2.P + e2*w.  Splitting the coefficient net at u = 1/2 (each column
// independently) gives the two halves' nets, whose hulls are tighter than the
// whole net's; likewise at v = 1/2 (each row).  If both halves of either split
// lie beyond +lim or below -lim for one plane, no evaluation point in [0,1]^2
// can meet the stop rule and Newton's outcome is "no hit".  Columns and rows
// stream from memory one at a time, so no 2D intermediate is held.
template <int M>
__device__ __forceinline__ void half_flags(const float (&a)[M + 1], const float (&b)[M + 1], const float (&w)[M + 1],
                                           float lim, bool (&f)[2][4]) {
    float ta[M + 1], tb[M + 1], tw[M + 1];
#pragma unroll
    for (int i = 0; i <= M; ++i) { ta[i] = a[i]; tb[i] = b[i]; tw[i] = w[i]; }
    auto upd = [&](int h, float x, float y, float ww) {
        const float m = lim * ww;
        f[h][0] &= x > m; f[h][1] &= x < -m; f[h][2] &= y > m; f[h][3] &= y < -m;
    };
    upd(0, ta[0], tb[0], tw[0]);
    upd(1, ta[M], tb[M], tw[M]);
#pragma unroll
    for (int k = 1; k <= M; ++k) {
#pragma unroll
        for (int i = 0; i <= M - k; ++i) {
            ta[i] = 0.5f * (ta[i] + ta[i + 1]);
            tb[i] = 0.5f * (tb[i] + tb[i + 1]);
            tw[i] = 0.5f * (tw[i] + tw[i + 1]);
        }
        upd(0, ta[0], tb[0], tw[0]);              // k-th point of the lower half
        upd(1, ta[M - k], tb[M - k], tw[M - k]);  // of the upper half
    }
}

template <int P, int Q>
__device__ __forceinline__ bool subdiv_misses(const float* __restrict__ blk, const RayFrame& r, const PatchRay& pr,
                                              float lim) {
    constexpr int NP = padded_points(P, Q);
    auto coeff = [&](int k, float& a, float& b, float& w) {
        const float2 xy = __ldg(reinterpret_cast<const float2*>(blk) + k);
        const float2 zw = __ldg(reinterpret_cast<const float2*>(blk + 2 * NP) + k);
        const float x = xy.x, y = xy.y, z = zw.x;
        w = zw.y;
        a = fmaf(r.n1x, x, fmaf(r.n1y, y, fmaf(r.n1z, z, pr.e1 * w)));
        b = fmaf(r.n2x, x, fmaf(r.n2y, y, fmaf(r.n2z, z, pr.e2 * w)));
    };
    bool fu[2][4] = {{true, true, true, true}, {true, true, true, true}};
#pragma unroll 1
    for (int j = 0; j <= Q; ++j) {  // split every column at u = 1/2
        float a[P + 1], b[P + 1], w[P + 1];
#pragma unroll
        for (int i = 0; i <= P; ++i) coeff(i * (Q + 1) + j, a[i], b[i], w[i]);
        half_flags<P>(a, b, w, lim, fu);
    }
    if ((fu[0][0] | fu[0][1] | fu[0][2] | fu[0][3]) && (fu[1][0] | fu[1][1] | fu[1][2] | fu[1][3])) return true;
    bool fv[2][4] = {{true, true, true, true}, {true, true, true, true}};
#pragma unroll 1
    for (int i = 0; i <= P; ++i) {  // split every row at v = 1/2
        float a[Q + 1], b[Q + 1], w[Q + 1];
#pragma unroll
        for (int j = 0; j <= Q; ++j) coeff(i * (Q + 1) + j, a[j], b[j], w[j]);
        half_flags<Q>(a, b, w, lim, fv);
    }
    return (fv[0][0] | fv[0][1] | fv[0][2] | fv[0][3]) && (fv[1][0] | fv[1][1] | fv[1][2] | fv[1][3]);
}

// Exact ray-space hull test ("clip" cull).  With w > 0, (r1, r2)(u,v) =
// (sum B_i a_i, sum B_i b_i) / sum B_i w_i, where (a_i, b_i) = (n1.P_i + e1 w_i,
// n2.P_i + e2 w_i) are the homogeneous plane residuals of the control points.
// If a unit direction d has d.(a_i, b_i) > M for every point, with
// M = lim * max_i w_i, then d.(r1, r2) > lim everywhere on [0,1]^2, hence
// |r1| + |r2| > lim >= eps and Newton cannot converge: the (ray, patch) test
// is skipped without changing any result.  Such a d exists iff the origin lies
// outside the convex hull of the points (up to the margin).
//
// Pass 1 keeps the arc of directions d with d.p > 0 for every point seen so
// far: it starts as the half circle around the first point and each further
// point either leaves it, trims one end to the point's perpendicular, or
// empties it (origin inside the hull).  This is the exact 2D hull test in
// O(points).  Pass 2 takes the arc's bisector and checks d.p_i > M |d| for
// every point, so rounding in pass 1 can only cost a cull, never cause a
// wrong one.  Subdividing the residual nets at u = 1/2 or v = 1/2 (de
// Casteljau averages) tightens the hulls: a pair is also culled when both
// halves' hulls miss the origin.
struct Arc {
    float rx, ry, lx, ly;  // clockwise and counter-clockwise ends of the arc of separating directions
    int st;                // 0: no point yet, 1: arc non-empty, 2: empty (no separating direction)
};

__device__ __forceinline__ void arc_add(Arc& A, float px, float py) {
    if (A.st == 1) {
        const float sR = fmaf(A.rx, px, A.ry * py), sL = fmaf(A.lx, px, A.ly * py);
        if (sR > 0.f) {
            if (!(sL > 0.f)) { A.lx = -py; A.ly = px; }
        } else if (sL > 0.f) {
            A.rx = py; A.ry = -px;
        } else {
            A.st = 2;  // both ends outside the point's half circle (or NaN): no direction left
        }
    } else if (A.st == 0) {
        A.rx = py; A.ry = -px; A.lx = -py; A.ly = px;
        A.st = (px != 0.f || py != 0.f) ? 1 : 2;
    }
}

// Bisector of the arc (unnormalised) and the margin it must clear: M * |d|.
__device__ __forceinline__ bool arc_direction(const Arc& A, float M, float& dx, float& dy, float& need) {
    if (A.st != 1) return false;
    dx = A.rx + A.lx;
    dy = A.ry + A.ly;
    need = M * sqrtf(fmaf(dx, dx, dy * dy));
    return dx != 0.f || dy != 0.f;
}

template <int P, int Q>
__device__ __forceinline__ void residual_point(const float* __restrict__ blk, int k, const RayFrame& r,
                                               const PatchRay& pr, float& a, float& b, float& w) {
    constexpr int NP = padded_points(P, Q);
    const float2 xy = __ldg(reinterpret_cast<const float2*>(blk) + k);
    const float2 zw = __ldg(reinterpret_cast<const float2*>(blk + 2 * NP) + k);
    const float x = xy.x, y = xy.y, z = zw.x;
    w = zw.y;
    a = fmaf(r.n1x, x, fmaf(r.n1y, y, fmaf(r.n1z, z, pr.e1 * w)));
    b = fmaf(r.n2x, x, fmaf(r.n2y, y, fmaf(r.n2z, z, pr.e2 * w)));
}

// Depth 0: the whole net.  Returns true when the pair can be skipped; wmax
// gets the largest weight (the margin's scale for the subdivided test).
template <int P, int Q>
__device__ __forceinline__ bool clip_whole(const float* __restrict__ blk, const RayFrame& r, const PatchRay& pr,
                                           float lim, float& wmax) {
    constexpr int N = (P + 1) * (Q + 1);
    Arc A;
    A.st = 0;
    wmax = 0.f;
#pragma unroll 4
    for (int k = 0; k < N; ++k) {
        float a, b, w;
        residual_point<P, Q>(blk, k, r, pr, a, b, w);
        wmax = fmaxf(wmax, w);
        arc_add(A, a, b);
    }
    float dx, dy, need;
    if (!arc_direction(A, lim * wmax, dx, dy, need)) return false;
    bool sep = true;
#pragma unroll 4
    for (int k = 0; k < N; ++k) {
        float a, b, w;
        residual_point<P, Q>(blk, k, r, pr, a, b, w);
        sep &= fmaf(dx, a, dy * b) > need;
    }
    return sep;
}

// Both halves of a degree-M polygon at 1/2 from one de Casteljau triangle:
// lo holds the control values on t in [0, 1/2], hi those on [1/2, 1].
template <int M>
__device__ __forceinline__ void split_poly(const float (&c)[M + 1], float (&lo)[M + 1], float (&hi)[M + 1]) {
    float t[M + 1];
#pragma unroll
    for (int i = 0; i <= M; ++i) t[i] = c[i];
    lo[0] = t[0];
    hi[M] = t[M];
#pragma unroll
    for (int k = 1; k <= M; ++k) {
#pragma unroll
        for (int i = 0; i <= M - k; ++i) t[i] = 0.5f * (t[i] + t[i + 1]);
        lo[k] = t[0];
        hi[M - k] = t[M - k];
    }
}

// Depth 1: the two halves of the net split at u = 1/2 (ALONG_U) or at
// v = 1/2.  Every line of the net along the split direction is split on its
// own, so the halves' points stream out one line at a time and no 2D net is
// held in registers.  Returns true when both halves' hulls miss the origin.
template <int P, int Q, bool ALONG_U>
__device__ __forceinline__ bool clip_halves(const float* __restrict__ blk, const RayFrame& r, const PatchRay& pr,
                                            float M) {
    constexpr int D = ALONG_U ? P : Q;           // degree along the split
    constexpr int L = ALONG_U ? Q + 1 : P + 1;   // lines split
    auto line = [&](int l, float (&la)[D + 1], float (&lb)[D + 1], float (&ua)[D + 1], float (&ub)[D + 1]) {
        float a[D + 1], b[D + 1];
#pragma unroll
        for (int k = 0; k <= D; ++k) {
            float w;
            residual_point<P, Q>(blk, ALONG_U ? k * (Q + 1) + l : l * (Q + 1) + k, r, pr, a[k], b[k], w);
        }
        split_poly<D>(a, la, ua);
        split_poly<D>(b, lb, ub);
    };
    Arc A0, A1;
    A0.st = 0;
    A1.st = 0;
#pragma unroll 1
    for (int l = 0; l < L; ++l) {
        float la[D + 1], lb[D + 1], ua[D + 1], ub[D + 1];
        line(l, la, lb, ua, ub);
#pragma unroll
        for (int k = 0; k <= D; ++k) {
            arc_add(A0, la[k], lb[k]);
            arc_add(A1, ua[k], ub[k]);
        }
        if (A0.st == 2 || A1.st == 2) return false;  // a half whose hull holds the origin
    }
    float d0x, d0y, n0, d1x, d1y, n1;
    if (!arc_direction(A0, M, d0x, d0y, n0) || !arc_direction(A1, M, d1x, d1y, n1)) return false;
    bool sep = true;
#pragma unroll 1
    for (int l = 0; l < L && sep; ++l) {
        float la[D + 1], lb[D + 1], ua[D + 1], ub[D + 1];
        line(l, la, lb, ua, ub);
#pragma unroll
        for (int k = 0; k <= D; ++k)
            sep &= (fmaf(d0x, la[k], d0y * lb[k]) > n0) & (fmaf(d1x, ua[k], d1y * ub[k]) > n1);
    }
    return sep;
}

// The clip cull: the whole net, then its halves at u = 1/2, then at v = 1/2.
template <int P, int Q>
__device__ __forceinline__ bool clip_misses(const float* __restrict__ blk, const RayFrame& r, const PatchRay& pr,
                                            float lim) {
    float wmax;
    if (clip_whole<P, Q>(blk, r, pr, lim, wmax)) return true;
    const float M = lim * wmax;
    return clip_halves<P, Q, true>(blk, r, pr, M) || clip_halves<P, Q, false>(blk, r, pr, M);
}

// Oriented-box test of a (ray, patch) pair, before any work item is made.
// The box holds the dehomogenised control points, hence the patch (w > 0).
// It is widened by eps plus a rounding allowance for the FP32 projections, so
// a ray that misses it cannot come within eps of the patch: Newton could not
// converge there and the pair is dropped without changing any result.
// obb: (axis_k, half extent_k) for k = 0..2, then (centre, 0).
__device__ __forceinline__ bool obb_misses(const float4* __restrict__ obb, const RayFrame& r, float eps) {
    const float4 a0 = __ldg(obb), a1 = __ldg(obb + 1), a2 = __ldg(obb + 2), c = __ldg(obb + 3);
    const float ox = r.ox - c.x, oy = r.oy - c.y, oz = r.oz - c.z;
    const float slack = eps + 1e-5f * (fabsf(ox) + fabsf(oy) + fabsf(oz) + a0.w + a1.w + a2.w);
    float tn = -INFINITY, tf = INFINITY;
    auto slab_k = [&](const float4 a) {
        const float o = fmaf(a.x, ox, fmaf(a.y, oy, a.z * oz));
        const float d = fmaf(a.x, r.dx, fmaf(a.y, r.dy, a.z * r.dz));
        const float h = a.w + slack;
        const float id = 1.f / d;
        const float t0 = (-h - o) * id, t1 = (h - o) * id;
        if (t0 == t0 && t1 == t1) {  // a NaN (d = 0 exactly on the boundary, or a NaN ray) constrains nothing
            tn = fmaxf(tn, fminf(t0, t1));
            tf = fminf(tf, fmaxf(t0, t1));
        }
    };
    slab_k(a0);
    slab_k(a1);
    slab_k(a2);
    return tf < tn;
}

// FP64 refinement of a converged (u, v): the ray's planes are rebuilt in
// double from the (float) ray (the FP32 planes are off the ray by an
// ulp-sized angle, which a grazing ray turns into a t shift), then up to 16
// Newton steps in double (a ray that nearly touches the surface has two
// crossings close together, where Newton converges only linearly), each
// re-evaluating the patch, for as long as the residual decreases (a full step,
// else a half, quarter or eighth of it); the point with the smallest residual
// is kept, so the step never makes a converged FP32 hit worse.  A step below 1e-7 in (u, v) ends the
// refinement with a first-order move of S (no further evaluation): that is
// the common case, one FP64 evaluation per hit.  S, dS/du, dS/dv and t are
// those of the final (u, v), in double.  Not inlined: every caller (Newton on
// convergence, the wavefront's resolve from a recorded (u, v)) runs the same
// machine code, so the result depends on nothing but (u, v) and the ray.
template <int P, int Q>
__device__ __noinline__ void final_step_fp64(const float* __restrict__ blk, const RayFrame& r, const PatchRay& pr,
                                             NewtonOut& o) {
    const double dx = r.dx, dy = r.dy, dz = r.dz;
    const double ax = fabs(dx), ay = fabs(dy), az = fabs(dz);
    double n1[3], n2[3];
    if (ax > ay && ax > az) {
        const double l = sqrt(dx * dx + dy * dy);
        n1[0] = dy / l; n1[1] = -dx / l; n1[2] = 0.0;
    } else {
        const double l = sqrt(dy * dy + dz * dz);
        n1[0] = 0.0; n1[1] = dz / l; n1[2] = -dy / l;
    }
    const double il = 1.0 / sqrt(dx * dx + dy * dy + dz * dz);
    const double ux = dx * il, uy = dy * il, uz = dz * il;
    n2[0] = n1[1] * uz - n1[2] * uy;
    n2[1] = n1[2] * ux - n1[0] * uz;
    n2[2] = n1[0] * uy - n1[1] * ux;
    const double oc[3] = {pr.ocx, pr.ocy, pr.ocz};
    const double e1 = -(n1[0] * oc[0] + n1[1] * oc[1] + n1[2] * oc[2]);
    const double e2 = -(n2[0] * oc[0] + n2[1] * oc[1] + n2[2] * oc[2]);
    double u = o.u, v = o.v;
    double H[4], Hu[4], Hv[4], S[3], Su[3], Sv[3];
    auto eval = [&]() {
        eval_patch_fp64<P, Q>(blk, u, v, H, Hu, Hv);
        const double iw = 1.0 / H[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            S[a] = H[a] * iw;
            Su[a] = (Hu[a] - S[a] * Hu[3]) * iw;
            Sv[a] = (Hv[a] - S[a] * Hv[3]) * iw;
        }
    };
    auto residual = [&](double& r1, double& r2) {
        r1 = n1[0] * S[0] + n1[1] * S[1] + n1[2] * S[2] + e1;
        r2 = n2[0] * S[0] + n2[1] * S[1] + n2[2] * S[2] + e2;
        return fabs(r1) + fabs(r2);
    };
    eval();
    double r1, r2;
    double best = residual(r1, r2);
    double bu = u, bv = v, bS[3] = {S[0], S[1], S[2]}, bSu[3] = {Su[0], Su[1], Su[2]}, bSv[3] = {Sv[0], Sv[1], Sv[2]};
#pragma unroll 1
    for (int it = 0; it < 16 && best > 0.0; ++it) {
        const double j11 = n1[0] * Su[0] + n1[1] * Su[1] + n1[2] * Su[2];
        const double j21 = n2[0] * Su[0] + n2[1] * Su[1] + n2[2] * Su[2];
        const double j12 = n1[0] * Sv[0] + n1[1] * Sv[1] + n1[2] * Sv[2];
        const double j22 = n2[0] * Sv[0] + n2[1] * Sv[1] + n2[2] * Sv[2];
        const double det = j11 * j22 - j12 * j21;
        if (det == 0.0) break;
        const double du = (j22 * r1 - j12 * r2) / det, dv = (j11 * r2 - j21 * r1) / det;
        const double u_at = u, v_at = v;
        const double un = fmin(fmax(u - du, 0.0), 1.0), vn = fmin(fmax(v - dv, 0.0), 1.0);
        if (fabs(un - u) + fabs(vn - v) < 1e-7) {
            // a small step: its second-order remainder is below float resolution, so the point
            // moves to first order without another evaluation
            const double su = un - u, sv = vn - v;
            u = un;
            v = vn;
#pragma unroll
            for (int a = 0; a < 3; ++a) S[a] += Su[a] * su + Sv[a] * sv;
            bu = u; bv = v;
#pragma unroll
            for (int a = 0; a < 3; ++a) { bS[a] = S[a]; bSu[a] = Su[a]; bSv[a] = Sv[a]; }
            break;
        }
        // the full step, else half, quarter and eighth steps (backtracking): a grazing ray's
        // residual is far from linear over a full step, and a shorter one still makes progress
        bool progress = false;
        double lam = 1.0;
#pragma unroll 1
        for (int half = 0; half < 4 && !progress; ++half, lam *= 0.5) {
            u = fmin(fmax(u_at - lam * du, 0.0), 1.0);
            v = fmin(fmax(v_at - lam * dv, 0.0), 1.0);
            eval();
            const double res = residual(r1, r2);
            if (res < best) {
                progress = true;
                best = res;
                bu = u; bv = v;
#pragma unroll
                for (int a = 0; a < 3; ++a) { bS[a] = S[a]; bSu[a] = Su[a]; bSv[a] = Sv[a]; }
            }
        }
        if (!progress) break;  // keep the best point so far
    }
    u = bu; v = bv;
#pragma unroll
    for (int a = 0; a < 3; ++a) { S[a] = bS[a]; Su[a] = bSu[a]; Sv[a] = bSv[a]; }
    const double t = (S[0] - oc[0]) * dx + (S[1] - oc[1]) * dy + (S[2] - oc[2]) * dz;
    o.u = (float)u;
    o.v = (float)v;
    o.t = (float)t;
    o.sx = (float)S[0]; o.sy = (float)S[1]; o.sz = (float)S[2];
    o.ux = (float)Su[0]; o.uy = (float)Su[1]; o.uz = (float)Su[2];
    o.vx = (float)Sv[0]; o.vy = (float)Sv[1]; o.vz = (float)Sv[2];
    o.fp64_final = 1;
}

// The ray's two planes rebuilt in double from the (float) ray, as the FP64
// oracle forms them (MathUtils::getRayPlanes, src/math/math_utils.h:33-54, in
// double), with the offsets of the patch-local frame.
struct PlanesF64 {
    double n1[3], n2[3], e1, e2;
};
__device__ __forceinline__ PlanesF64 planes_fp64(const RayFrame& r, const PatchRay& pr) {
    const double dx = r.dx, dy = r.dy, dz = r.dz;
    const double ax = fabs(dx), ay = fabs(dy), az = fabs(dz);
    PlanesF64 p;
    if (ax > ay && ax > az) {
        const double l = sqrt(dx * dx + dy * dy);
        p.n1[0] = dy / l; p.n1[1] = -dx / l; p.n1[2] = 0.0;
    } else {
        const double l = sqrt(dy * dy + dz * dz);
        p.n1[0] = 0.0; p.n1[1] = dz / l; p.n1[2] = -dy / l;
    }
    const double il = 1.0 / sqrt(dx * dx + dy * dy + dz * dz);
    const double ux = dx * il, uy = dy * il, uz = dz * il;
    p.n2[0] = p.n1[1] * uz - p.n1[2] * uy;
    p.n2[1] = p.n1[2] * ux - p.n1[0] * uz;
    p.n2[2] = p.n1[0] * uy - p.n1[1] * ux;
    p.e1 = -(p.n1[0] * pr.ocx + p.n1[1] * pr.ocy + p.n1[2] * pr.ocz);
    p.e2 = -(p.n2[0] * pr.ocx + p.n2[1] * pr.ocy + p.n2[2] * pr.ocz);
    return p;
}

// FP64 continuation of a Newton solve whose FP32 residual fell into the
// decision band at evaluation `it`: the same iteration (residual test, seeded
// pull on a singular Jacobian, adjugate step, clamping; the seed sequence
// continues where the FP32 loop left it) runs in double from the current
// (u, v) for the evaluations left of max_iter, starting by re-evaluating the
// current point in double.  Near eps the FP32 residual is at its rounding
// floor on patches with extreme weights (its error is of the order of eps),
// so the stop rule is applied to the FP64 residual: the solve converges, or
// not, where the same method in double does.  Not inlined: it runs only in the
// band, and keeps its double registers out of the FP32 loop.
template <int P, int Q>
__device__ __noinline__ void newton_tail_fp64(const float* __restrict__ blk, const RayFrame& r, const PatchRay& pr,
                                              float u0f, float v0f, float uf, float vf, int it, uint32_t seed,
                                              const NewtonOpts& op, NewtonOut& o) {
    const PlanesF64 pl = planes_fp64(r, pr);
    const double u0 = u0f, v0 = v0f, eps = op.eps, det_eps = op.det_eps;
    double u = uf, v = vf;
    for (; it <= op.max_iter; ++it) {
        double H[4], Hu[4], Hv[4], S[3], Su[3], Sv[3];
        eval_patch_fp64<P, Q>(blk, u, v, H, Hu, Hv);
        ++o.fp64_solves;
        const double iw = 1.0 / H[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            S[a] = H[a] * iw;
            Su[a] = (Hu[a] - S[a] * Hu[3]) * iw;
            Sv[a] = (Hv[a] - S[a] * Hv[3]) * iw;
        }
        const double r1 = pl.n1[0] * S[0] + pl.n1[1] * S[1] + pl.n1[2] * S[2] + pl.e1;
        const double r2 = pl.n2[0] * S[0] + pl.n2[1] * S[1] + pl.n2[2] * S[2] + pl.e2;
        if (fabs(r1) + fabs(r2) < eps) {
            o.evals = it;
            o.u = (float)u; o.v = (float)v;
            o.sx = (float)S[0]; o.sy = (float)S[1]; o.sz = (float)S[2];
            o.ux = (float)Su[0]; o.uy = (float)Su[1]; o.uz = (float)Su[2];
            o.vx = (float)Sv[0]; o.vy = (float)Sv[1]; o.vz = (float)Sv[2];
            o.t = (float)((S[0] - pr.ocx) * r.dx + (S[1] - pr.ocy) * r.dy + (S[2] - pr.ocz) * r.dz);
            return;
        }
        const double j11 = pl.n1[0] * Su[0] + pl.n1[1] * Su[1] + pl.n1[2] * Su[2];
        const double j21 = pl.n2[0] * Su[0] + pl.n2[1] * Su[1] + pl.n2[2] * Su[2];
        const double j12 = pl.n1[0] * Sv[0] + pl.n1[1] * Sv[1] + pl.n1[2] * Sv[2];
        const double j22 = pl.n2[0] * Sv[0] + pl.n2[1] * Sv[1] + pl.n2[2] * Sv[2];
        seed = pcg_hash(seed);
        const double rnd1 = (double)seed * 2.3283064365386963e-10;
        seed = pcg_hash(seed);
        const double rnd2 = (double)seed * 2.3283064365386963e-10;
        const double det = j11 * j22 - j12 * j21;
        if (fabs(det) < det_eps) {
            u = u + 0.1 * ((u0 - u) * rnd1);
            v = v + 0.1 * ((v0 - v) * rnd2);
        } else {
            u = u - (j22 * r1 - j12 * r2) / det;
            v = v - (j11 * r2 - j21 * r1) / det;
        }
        u = fmin(fmax(u, 0.0), 1.0);
        v = fmin(fmax(v, 0.0), 1.0);
    }
    o.evals = -op.max_iter;
    o.u = (float)u;
    o.v = (float)v;
}

// Newton-Raphson on F(u,v) = (n1.S + e1, n2.S + e2) from (u0, v0); the
// iteration, thresholds, seeded pull on a singular Jacobian and clamping follow
// BezierPatchOps::newtonRhapson (src/math/bezier_patch.h:197-266).  When
// cond_fp64 > 0 and ||J||_F^2 / |det J| exceeds it, the 2x2 solve is done in
// FP64 (products of floats are exact there, so det J has no cancellation).
// With op.fp64_band (the FP64 final-step mode) convergence within the
// decision band around eps is decided in FP64 (newton_tail_fp64).  FINAL = false compiles the FP64 final step and the FP64
// decisions out (for kernels that run without them, so that they carry no
// call to them).
//
// The solve is a state machine advanced one evaluation at a time
// (newton_step), so that a kernel can run the evaluations of many solves in
// lockstep and give a lane a new solve as soon as its own ends; newton() runs
// one solve to its end.  One early exit is added, exact: when a regular
// Newton step (not the seeded pull) leaves the clamped iterate unchanged, the
// next evaluation would repeat this one, with the same residual and step,
// until the budget runs out, so the solve ends there unconverged (evals counts
// the evaluations actually run; the outcome, -max_iter, is unchanged).
struct NewtonState {
    float u, v, u0, v0;
    uint32_t seed;
    int it;      // the evaluation about to run, 1-based
    int done;    // evaluations run
    int f64;     // 2x2 steps solved in FP64 so far
    int fp64;    // 1: the solve ended in the decision band; FP64 continues from (u, v) at
                 // evaluation it (newton_finish)
};

__device__ __forceinline__ NewtonState newton_start(float u0, float v0, uint32_t seed) {
    NewtonState s;
    s.u = u0; s.v = v0; s.u0 = u0; s.v0 = v0;
    s.seed = seed;
    s.it = 1;
    s.done = 0;
    s.f64 = 0;
    s.fp64 = 0;
    return s;
}

// One evaluation (and step) of the solve in s.  Returns true when the solve
// has ended, with o holding its FP32 outcome (o is written only then); the
// FP64 work that decides or refines it is left to newton_finish, so that the
// evaluation loop makes no calls.
template <int P, int Q, bool FINAL = true>
__device__ __forceinline__ bool newton_step(const float* __restrict__ blk, const RayFrame& r, const PatchRay& pr,
                                            NewtonState& s, const NewtonOpts& op, NewtonOut& o) {
    const bool band = FINAL && op.fp64_band;
    const float accept = band ? kBandLo * op.eps : op.eps;
    auto end = [&]() {
        o.fp64_solves = s.f64;
        o.flat = 0;
        o.fp64_final = 0;
        o.done = s.done;
    };
    if (s.it > op.max_iter) {  // no evaluation left (max_iter <= 0)
        end();
        o.evals = -op.max_iter;
        o.u = s.u; o.v = s.v;
        return true;
    }
    const float u = s.u, v = s.v;
    float H[4], Hu[4], Hv[4];
    eval_patch<P, Q>(blk, u, v, H, Hu, Hv);
    ++s.done;
    const float iw = __frcp_rn(H[3]);
    const float sx = H[0] * iw, sy = H[1] * iw, sz = H[2] * iw;
    const float ux = (Hu[0] - sx * Hu[3]) * iw, uy = (Hu[1] - sy * Hu[3]) * iw, uz = (Hu[2] - sz * Hu[3]) * iw;
    const float vx = (Hv[0] - sx * Hv[3]) * iw, vy = (Hv[1] - sy * Hv[3]) * iw, vz = (Hv[2] - sz * Hv[3]) * iw;
    const float r1 = fmaf(r.n1x, sx, fmaf(r.n1y, sy, fmaf(r.n1z, sz, pr.e1)));
    const float r2 = fmaf(r.n2x, sx, fmaf(r.n2y, sy, fmaf(r.n2z, sz, pr.e2)));
    const float res = fabsf(r1) + fabsf(r2);
    if (band && res >= accept && res < kBandHi * op.eps) {
        end();
        s.fp64 = 1;  // FP64 continues from (u, v) at this evaluation
        return true;
    }
    if (res < accept) {
        end();
        o.evals = s.it;
        o.u = u; o.v = v;
        o.sx = sx; o.sy = sy; o.sz = sz;
        o.ux = ux; o.uy = uy; o.uz = uz;
        o.vx = vx; o.vy = vy; o.vz = vz;
        o.t = fmaf(sx, r.dx, fmaf(sy, r.dy, fmaf(sz, r.dz, pr.tc)));
        return true;
    }
    const float j11 = r.n1x * ux + r.n1y * uy + r.n1z * uz;
    const float j21 = r.n2x * ux + r.n2y * uy + r.n2z * uz;
    const float j12 = r.n1x * vx + r.n1y * vy + r.n1z * vz;
    const float j22 = r.n2x * vx + r.n2y * vy + r.n2z * vz;
    s.seed = pcg_hash(s.seed);
    const float rnd1 = (float)s.seed * 2.3283064e-10f;
    s.seed = pcg_hash(s.seed);
    const float rnd2 = (float)s.seed * 2.3283064e-10f;
    const float det = j11 * j22 - j12 * j21;
    float un, vn;
    const bool pull = fabsf(det) < op.det_eps;
    if (pull) {
        un = u + 0.1f * ((s.u0 - u) * rnd1);
        vn = v + 0.1f * ((s.v0 - v) * rnd2);
    } else if (op.cond_fp64 > 0.f &&
               (j11 * j11 + j12 * j12 + j21 * j21 + j22 * j22) > op.cond_fp64 * fabsf(det)) {
        const double dd = (double)j11 * j22 - (double)j12 * j21;
        un = (float)((double)u - ((double)j22 * r1 - (double)j12 * r2) / dd);
        vn = (float)((double)v - ((double)j11 * r2 - (double)j21 * r1) / dd);
        ++s.f64;
    } else {
        const float id = __frcp_rn(det);
        un = u - (j22 * r1 - j12 * r2) * id;
        vn = v - (j11 * r2 - j21 * r1) * id;
    }
    s.u = fminf(fmaxf(un, 0.f), 1.f);
    s.v = fminf(fmaxf(vn, 0.f), 1.f);
    ++s.it;
    const bool stuck = !pull && s.u == u && s.v == v;  // a fixed point of the iteration
    if (s.it > op.max_iter || stuck) {
        end();
        o.evals = -op.max_iter;
        o.u = s.u; o.v = s.v;
        return true;
    }
    return false;
}

// The FP64 part of an ended solve: the FP64 continuation newton_step asked
// for, then, when converged and op.fp64_final, the FP64 refinement of the point.
template <int P, int Q>
__device__ __forceinline__ void newton_finish(const float* __restrict__ blk, const RayFrame& r, const PatchRay& pr,
                                              const NewtonState& s, const NewtonOpts& op, NewtonOut& o) {
    if (s.fp64 == 1) newton_tail_fp64<P, Q>(blk, r, pr, s.u0, s.v0, s.u, s.v, s.it, s.seed, op, o);
    if (o.evals > 0 && op.fp64_final) final_step_fp64<P, Q>(blk, r, pr, o);
}

template <int P, int Q, bool FINAL = true>
__device__ __forceinline__ NewtonOut newton(const float* __restrict__ blk, const RayFrame& r, const PatchRay& pr,
                                            float u0, float v0, uint32_t seed, const NewtonOpts& op) {
    NewtonOut o;
    NewtonState s = newton_start(u0, v0, seed);
    while (!newton_step<P, Q, FINAL>(blk, r, pr, s, op, o)) {
    }
    if (FINAL) newton_finish<P, Q>(blk, r, pr, s, op, o);
    return o;
}

// The reference's ray/bilinear-patch guess through the four corners
// (BezierPatchOps::biliniearRay, src/math/bezier_patch.h:272-327), computed in
// world coordinates with round-to-nearest products and sums that are never
// fused, so it reproduces the reference's host arithmetic exactly.  As written
// there, n.pb and n.d vanish up to rounding (n = d x pb), so the guess is
// (0.5, 0.5) unless that rounding noise selects a root.
__device__ __forceinline__ void bilinear_guess(const float4* __restrict__ cr, const RayFrame& r, float& gu,
                                               float& gv) {
#define M_(a, b) __fmul_rn(a, b)
#define A_(a, b) __fadd_rn(a, b)
#define S_(a, b) __fsub_rn(a, b)
    const float4 c00 = __ldg(cr), c10 = __ldg(cr + 1), c11 = __ldg(cr + 2), c01 = __ldg(cr + 3);
    float e10[3] = {S_(c10.x, c00.x), S_(c10.y, c00.y), S_(c10.z, c00.z)};
    float e11[3] = {S_(c11.x, c10.x), S_(c11.y, c10.y), S_(c11.z, c10.z)};
    float e00[3] = {S_(c01.x, c00.x), S_(c01.y, c00.y), S_(c01.z, c00.z)};
    float w[3] = {S_(c01.x, c11.x), S_(c01.y, c11.y), S_(c01.z, c11.z)};
    auto cross = [](const float* a, const float* b, float* o) {
        o[0] = S_(M_(a[1], b[2]), M_(a[2], b[1]));
        o[1] = S_(M_(a[2], b[0]), M_(a[0], b[2]));
        o[2] = S_(M_(a[0], b[1]), M_(a[1], b[0]));
    };
    auto dot = [](const float* a, const float* b) { return A_(A_(M_(a[0], b[0]), M_(a[1], b[1])), M_(a[2], b[2])); };
    float qn[3];
    cross(e10, w, qn);
    const float d[3] = {r.dx, r.dy, r.dz};
    float q00[3] = {S_(c00.x, r.ox), S_(c00.y, r.oy), S_(c00.z, r.oz)};
    float q10[3] = {S_(c10.x, r.ox), S_(c10.y, r.oy), S_(c10.z, r.oz)};
    float t0[3], t1[3];
    cross(q00, d, t0);
    cross(q10, d, t1);
    const float a = dot(t0, e00), c = dot(qn, d);
    float b = dot(t1, e11);
    b = S_(b, A_(a, c));
    float det = S_(M_(b, b), M_(M_(4.0f, a), c));
    gu = 0.5f;
    gv = 0.5f;
    if (det < 0.f) return;
    det = __fsqrt_rn(det);
    float ux[2];
    if (c == 0.f) { ux[0] = __fdiv_rn(-a, b); ux[1] = -1.f; }
    else {
        ux[0] = __fdiv_rn(S_(-b, copysignf(det, b)), 2.0f);
        ux[1] = __fdiv_rn(a, ux[0]);
        ux[0] = __fdiv_rn(ux[0], c);
    }
    float best = INFINITY;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        if (ux[i] < 0.f || ux[i] > 1.f) continue;
        const float om = S_(1.0f, ux[i]);
        const float pb[3] = {A_(M_(e00[0], om), M_(e11[0], ux[i])), A_(M_(e00[1], om), M_(e11[1], ux[i])),
                             A_(M_(e00[2], om), M_(e11[2], ux[i]))};
        float n[3];
        cross(d, pb, n);
        const float dd = dot(n, n), tx = dot(n, pb), vx = dot(n, d);
        if (tx > 0.f && 0.f <= vx && vx <= dd && tx < best) {
            gu = ux[i];
            gv = __fdiv_rn(vx, dd);
            best = tx;
        }
    }
#undef M_
#undef A_
#undef S_
}

// Slab test returning the entry distance (tmin starts at 0) or +inf, as
// BoundsOps::intersectBound (src/math/bounds_ops.h:83-114).
__device__ __forceinline__ float slab(float lox, float loy, float loz, float hix, float hiy, float hiz,
                                      const RayFrame& r, float rdx, float rdy, float rdz) {
    const float t0x = (lox - r.ox) * rdx, t1x = (hix - r.ox) * rdx;
    const float t0y = (loy - r.oy) * rdy, t1y = (hiy - r.oy) * rdy;
    const float t0z = (loz - r.oz) * rdz, t1z = (hiz - r.oz) * rdz;
    const float lo = fmaxf(fminf(t0z, t1z), fmaxf(fminf(t0y, t1y), fmaxf(fminf(t0x, t1x), 0.f)));
    const float hi = fminf(fmaxf(t0z, t1z), fminf(fmaxf(t0y, t1y), fmaxf(t0x, t1x)));
    return (lo <= hi && hi > 0.f) ? lo : INFINITY;
}

}  // namespace dev
}  // namespace nrt
