// refine_math.h -- the curvature refinement's per-span arithmetic, shared by
// the host refinement (refine.cpp) and the device one (refine_dev.cu): the
// number of knots to insert into one knot span of one curve of the net, as
// NurbsOps::knotsToAdd (src/math/nurbs.h:254-281) counts them,
//     floor( C * max_j |A_j| * (U_i+1 - U_i)^1.5 / sqrt( sum_j |V_j| / p ) )
// with V_j = p (P_j - P_j-1) / (U_j+p - U_j) the first-derivative control
// vectors of the span and A_j = (p-1) (V_j - V_j-1) / (U_j+p-1 - U_j) the
// second-derivative ones.  One rounding per operation (host -ffp-contract=off,
// device -fmad=false), correctly rounded division and square root on both.
// The power 1.5 is the host library's powf on the host (the reference's own
// call) and, on the device, x * sqrt(x) formed in double and rounded once to
// float (the correctly rounded x^1.5 but for inputs within 2^-29 of a
// rounding boundary).
#pragma once

#include <cmath>

#include "nrt_internal.h"

#ifdef __CUDACC__
#define NRT_RHD __host__ __device__
#else
#define NRT_RHD
#endif

namespace nrt {
namespace refine_math {

struct V3 {
    float x, y, z;
};

NRT_RHD inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
NRT_RHD inline V3 scale(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
NRT_RHD inline float norm(V3 a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }

NRT_RHD inline float pow15(float x) {
#ifdef __CUDA_ARCH__
    const double d = (double)x;
    return (float)(d * sqrt(d));
#else
    return powf(x, 1.5f);
#endif
}

// Algorithm A2.1: the span index of u in U (n+1 control points, degree p).
NRT_RHD inline int find_span(int n, int p, float u, const float* U) {
    if (u == U[n + 1]) return n;
    int lo = p, hi = n + 1, mid = (lo + hi) / 2;
    while (u < U[mid] || u >= U[mid + 1]) {
        if (u < U[mid]) hi = mid;
        else lo = mid;
        mid = (lo + hi) / 2;
    }
    return mid;
}

// How many times u occurs at or below index k.
NRT_RHD inline int multiplicity_at(const float* U, int k, float u) {
    int s = 0;
    for (int i = k; i >= 0 && U[i] == u; --i) ++s;
    return s;
}

// Knots to insert into span i (U[i] <= u < U[i+1]) of a curve of degree p;
// point(j) gives its j-th dehomogenised control point.
template <class PointAt>
NRT_RHD inline int knot_count(PointAt point, const float* U, int i, float C, int p) {
    V3 Vj[NRT_MAX_DEGREE + 1];
    float vsum = 0.f;
    const int base = i - p + 1;
    for (int j = base; j <= i; ++j) {
        const float d = U[j + p] - U[j];
        Vj[j - base] = d > 0.f ? scale(sub(point(j), point(j - 1)), p / d) : V3{0.f, 0.f, 0.f};
        vsum += norm(Vj[j - base]);
    }
    float amax = 0.f;
    for (int j = base + 1; j <= i; ++j) {
        const float d = U[j + p - 1] - U[j];
        const V3 A = d > 0.f ? scale(sub(Vj[j - base], Vj[j - 1 - base]), (p - 1) / d) : V3{0.f, 0.f, 0.f};
        amax = fmaxf(amax, norm(A));
    }
    const float num = amax * pow15(U[i + 1] - U[i]);
    const float den = sqrtf(vsum / p);
    if (!(den > 1e-9f)) return 0;
    const float nf = C * num / den;
    if (!(nf > 1e-9f)) return 0;
    return nf < (float)(1 << 20) ? (int)nf : (1 << 20);
}

}  // namespace refine_math
}  // namespace nrt
