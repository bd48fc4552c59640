// slot_pack.cuh -- what a scene stores per patch slot (the SoA control-point
// block, header, centre, corners, flatness, learned-guess frame and oriented
// box), computed by one function that the host builder (engine.cu) and the
// device builder (scene_build.cu) both call, so the two scenes hold the same
// bits.  Same arithmetic rules as scene_math.h: one rounding per operation
// (no contraction on either side), correctly rounded division and square
// root, no transcendental functions.
#pragma once

#include <cuda_runtime.h>

#include "device_scene.cuh"
#include "scene_math.h"

namespace nrt {

// std::min / std::max for doubles, spelled out (a NaN second argument keeps the first)
NRT_HD inline double dmin(double a, double b) { return (b < a) ? b : a; }
NRT_HD inline double dmax(double a, double b) { return (a < b) ? b : a; }

// Flatness of a patch: largest distance from a control point to the bilinear
// interpolation of the four corners at its (i/p, j/q) node; patchDelta,
// src/core/main.cpp:18-43.
NRT_HD inline float patch_delta(const float* P, int p, int q) {
    const int row = q + 1;
    float c00[3], c10[3], c01[3], c11[3];
    const int ci[4] = {0, p * row, q, p * row + q};
    float* co[4] = {c00, c10, c01, c11};
    for (int c = 0; c < 4; ++c) {
        const float iw = 1.0f / P[4 * ci[c] + 3];
        for (int k = 0; k < 3; ++k) co[c][k] = P[4 * ci[c] + k] * iw;
    }
    float d = 0.f;
    for (int i = 0; i <= p; ++i)
        for (int j = 0; j <= q; ++j) {
            const float u = (float)i / p, v = (float)j / q;
            const float a = (1 - u) * (1 - v), b = u * (1 - v), c = (1 - u) * v, e = u * v;
            const float* X = P + 4 * (i * row + j);
            const float iw = 1.0f / X[3];
            float s = 0.f;
            for (int k = 0; k < 3; ++k) {
                const float Pk = X[k] * iw;
                const float B = a * c00[k] + b * c10[k] + c * c01[k] + e * c11[k];
                s += (Pk - B) * (Pk - B);
            }
            d = fmaxf(d, sqrtf(s));
        }
    return d;
}

// Oriented bounding box of a patch's dehomogenised control points (their
// convex hull holds the patch when every weight is positive): axes from the
// principal directions of the points (cyclic Jacobi on the 3x3 covariance, in
// double, each rotation from the tangent formula of Golub & Van Loan's
// symmetric Schur step, 8.4.2), extents from the points' projections.  Four
// float4 per slot: (axis_k, half extent_k) for k = 0..2, then (centre, 0).  A
// patch with a non-positive weight gets infinite extents, so that it is never
// culled.
NRT_HD inline void patch_obb(const float* P, int p, int q, float4 out[4]) {
    const int n = (p + 1) * (q + 1);
    double X[3 * (NRT_MAX_DEGREE + 1) * (NRT_MAX_DEGREE + 1)];
    bool pos = true;
    double m[3] = {0, 0, 0};
    for (int i = 0; i < n; ++i) {
        const double w = P[4 * i + 3];
        pos = pos && w > 0.0;
        for (int k = 0; k < 3; ++k) {
            X[3 * i + k] = w != 0.0 ? P[4 * i + k] / w : 0.0;
            m[k] += X[3 * i + k] / n;
        }
    }
    double A[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, V[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (int i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) A[a][b] += (X[3 * i + a] - m[a]) * (X[3 * i + b] - m[b]);
    for (int sweep = 0; sweep < 32; ++sweep) {
        const double off = fabs(A[0][1]) + fabs(A[0][2]) + fabs(A[1][2]);
        if (off <= 1e-300 + 1e-15 * (fabs(A[0][0]) + fabs(A[1][1]) + fabs(A[2][2]))) break;
        for (int a = 0; a < 2; ++a)
            for (int b = a + 1; b < 3; ++b) {
                if (A[a][b] == 0.0) continue;
                // J = [[c, s], [-s, c]] in the (a, b) plane zeroes A[a][b] of J^T A J
                const double tau = (A[b][b] - A[a][a]) / (2.0 * A[a][b]);
                const double t = fabs(tau) > 1e150 ? 0.5 / tau
                                 : tau >= 0.0     ? 1.0 / (tau + sqrt(1.0 + tau * tau))
                                                  : -1.0 / (-tau + sqrt(1.0 + tau * tau));
                const double c = 1.0 / sqrt(1.0 + t * t), s = t * c;
                for (int k = 0; k < 3; ++k) {  // A <- A J
                    const double ka = A[k][a], kb = A[k][b];
                    A[k][a] = c * ka - s * kb;
                    A[k][b] = s * ka + c * kb;
                }
                for (int k = 0; k < 3; ++k) {  // A <- J^T A
                    const double ak = A[a][k], bk = A[b][k];
                    A[a][k] = c * ak - s * bk;
                    A[b][k] = s * ak + c * bk;
                }
                for (int k = 0; k < 3; ++k) {  // V <- V J
                    const double ka = V[k][a], kb = V[k][b];
                    V[k][a] = c * ka - s * kb;
                    V[k][b] = s * ka + c * kb;
                }
            }
    }
    double ctr[3] = {m[0], m[1], m[2]}, half[3];
    for (int a = 0; a < 3; ++a) {
        // round the axis to float first: the device projects with the stored axis
        const float ax[3] = {(float)V[0][a], (float)V[1][a], (float)V[2][a]};
        double lo = 1e300, hi = -1e300;
        for (int i = 0; i < n; ++i) {
            const double t = ax[0] * (X[3 * i] - m[0]) + ax[1] * (X[3 * i + 1] - m[1]) + ax[2] * (X[3 * i + 2] - m[2]);
            lo = dmin(lo, t);
            hi = dmax(hi, t);
        }
        half[a] = 0.5 * (hi - lo);
        for (int k = 0; k < 3; ++k) ctr[k] += ax[k] * 0.5 * (lo + hi);
        out[a] = make_float4(ax[0], ax[1], ax[2], 0.f);
    }
    double cmax = 0.0;
    for (int k = 0; k < 3; ++k) cmax = dmax(cmax, fabs(ctr[k]));
    for (int a = 0; a < 3; ++a) {
        // extents cover the float-rounded centre and axes
        const double h = half[a] * (1.0 + 1e-6) + 4e-7 * cmax + 1e-30;
        out[a].w = pos ? (float)(h * (1.0 + 1e-6)) : INFINITY;
    }
    out[3] = make_float4((float)ctr[0], (float)ctr[1], (float)ctr[2], 0.f);
}

// Bernstein values B[0..n] and derivatives dB[0..n] at 1/2.
NRT_HD inline void bernstein_half(int n, double* B, double* dB) {
    double c = 1.0;
    for (int i = 0; i <= n; ++i) {
        B[i] = c / ldexp(1.0, n);
        c = c * (n - i) / (i + 1);
    }
    double cm = 1.0, Bm[NRT_MAX_DEGREE + 1];
    for (int i = 0; i < n; ++i) {
        Bm[i] = cm / ldexp(1.0, n - 1);
        cm = cm * (n - 1 - i) / (i + 1);
    }
    for (int i = 0; i <= n; ++i) dB[i] = n * ((i > 0 ? Bm[i - 1] : 0.0) - (i < n ? Bm[i] : 0.0));
}

// Frame of the learned guess's features (see mlp.cuh): the tangent frame of
// the patch at (u, v) = (1/2, 1/2), in patch-local coordinates.  Axes A = dS/du,
// B = dS/dv and the normal of A x B scaled by sqrt|A x B|; origin
// S(1/2, 1/2) - A/2 - B/2, so that a point's frame coordinates (s, t) are its
// (u, v) to first order (the iterate of one Newton step from the midpoint).
// Rational evaluation in double from the weighted-homogeneous points.
// Degenerate nets (collapsed tangents) fall back to the box, normalised.
NRT_HD inline dev::PatchFrame patch_frame(const float* P, int p, int q, double cx, double cy, double cz, const Box3& b) {
    double Bu[NRT_MAX_DEGREE + 1], dBu[NRT_MAX_DEGREE + 1], Bv[NRT_MAX_DEGREE + 1], dBv[NRT_MAX_DEGREE + 1];
    bernstein_half(p, Bu, dBu);
    bernstein_half(q, Bv, dBv);
    double H[4] = {0, 0, 0, 0}, Hu[4] = {0, 0, 0, 0}, Hv[4] = {0, 0, 0, 0};
    for (int i = 0; i <= p; ++i)
        for (int j = 0; j <= q; ++j) {
            const float* c = P + 4 * (i * (q + 1) + j);
            const double w = c[3];
            const double X[4] = {c[0] - w * cx, c[1] - w * cy, c[2] - w * cz, w};
            for (int k = 0; k < 4; ++k) {
                H[k] += Bu[i] * Bv[j] * X[k];
                Hu[k] += dBu[i] * Bv[j] * X[k];
                Hv[k] += Bu[i] * dBv[j] * X[k];
            }
        }
    double A[3], B[3], o[3];
    for (int k = 0; k < 3; ++k) {
        const double S = H[k] / H[3];
        A[k] = (Hu[k] - S * Hu[3]) / H[3];
        B[k] = (Hv[k] - S * Hv[3]) / H[3];
        o[k] = S - 0.5 * A[k] - 0.5 * B[k];
    }
    const double N[3] = {A[1] * B[2] - A[2] * B[1], A[2] * B[0] - A[0] * B[2], A[0] * B[1] - A[1] * B[0]};
    const double nn = sqrt(N[0] * N[0] + N[1] * N[1] + N[2] * N[2]);
    const double aa = A[0] * A[0] + A[1] * A[1] + A[2] * A[2], bb = B[0] * B[0] + B[1] * B[1] + B[2] * B[2];
    dev::PatchFrame f{};
    double M[3][3];  // columns A, B, N/sqrt|N|
    double scale;
    if (nn > 1e-9 * (aa + bb) && aa > 0 && bb > 0) {
        const double s = 1.0 / sqrt(nn);
        for (int k = 0; k < 3; ++k) { M[k][0] = A[k]; M[k][1] = B[k]; M[k][2] = N[k] * s; }
        scale = sqrt(dmax(aa, bb));
    } else {
        const double cc[3] = {cx, cy, cz};
        for (int k = 0; k < 3; ++k) {
            o[k] = (double)b.lo[k] - cc[k];
            for (int l = 0; l < 3; ++l) M[k][l] = k == l ? dmax((double)b.hi[k] - b.lo[k], 1e-12) : 0.0;
        }
        scale = dmax(dmax(M[0][0], M[1][1]), M[2][2]);
    }
    const double det = M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) -
                       M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
                       M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
    const double id = 1.0 / det;
    const double inv[9] = {(M[1][1] * M[2][2] - M[1][2] * M[2][1]) * id, (M[0][2] * M[2][1] - M[0][1] * M[2][2]) * id,
                           (M[0][1] * M[1][2] - M[0][2] * M[1][1]) * id, (M[1][2] * M[2][0] - M[1][0] * M[2][2]) * id,
                           (M[0][0] * M[2][2] - M[0][2] * M[2][0]) * id, (M[0][2] * M[1][0] - M[0][0] * M[1][2]) * id,
                           (M[1][0] * M[2][1] - M[1][1] * M[2][0]) * id, (M[0][1] * M[2][0] - M[0][0] * M[2][1]) * id,
                           (M[0][0] * M[1][1] - M[0][1] * M[1][0]) * id};
    f.ox = (float)o[0]; f.oy = (float)o[1]; f.oz = (float)o[2];
    for (int k = 0; k < 9; ++k) f.m[k] = (float)inv[k];
    double hmax = 0.0;  // half-thickness of the control net along the frame's h axis
    for (int i = 0; i <= p; ++i)
        for (int j = 0; j <= q; ++j) {
            const float* c = P + 4 * (i * (q + 1) + j);
            const double X[3] = {c[0] / (double)c[3] - cx, c[1] / (double)c[3] - cy, c[2] / (double)c[3] - cz};
            const double d3[3] = {X[0] - o[0], X[1] - o[1], X[2] - o[2]};
            hmax = dmax(hmax, fabs(inv[6] * d3[0] + inv[7] * d3[1] + inv[8] * d3[2]));
        }
    f.slab = (float)dmax(hmax, 1e-6);
    f.flat = (float)(hmax * sqrt(fabs(det)) / dmax(scale * scale, 1e-30));
    f.lo[0] = (float)(b.lo[0] - cx); f.lo[1] = (float)(b.lo[1] - cy); f.lo[2] = (float)(b.lo[2] - cz);
    f.hi_x = (float)(b.hi[0] - cx); f.hi_y = (float)(b.hi[1] - cy); f.hi_z = (float)(b.hi[2] - cz);
    return f;
}

// Everything one slot stores, for patch `patch_id` of surface `surf` with
// weighted-homogeneous points P (degree p, q) and box b, whose block (XY and
// ZW halves, patch_math.cuh) starts `off` floats into the scene's block
// array; blk points there.
NRT_HD inline void pack_slot(const float* P, int p, int q, const Box3& b, int patch_id, int surf, long long off,
                             float* blk, int4& hdr, double4& ctr, float4 corners[4], float& delta,
                             dev::PatchFrame& frame, float4 obb[4]) {
    const int n = (p + 1) * (q + 1), np = dev::padded_points(p, q);
    const double cx = 0.5 * ((double)b.lo[0] + b.hi[0]), cy = 0.5 * ((double)b.lo[1] + b.hi[1]),
                 cz = 0.5 * ((double)b.lo[2] + b.hi[2]);
    bool pos = true;
    double rad = 0.0, wmin = INFINITY, wmax = 0.0;
    for (int i = 0; i < n; ++i) {
        const double w = P[4 * i + 3];
        pos = pos && (w > 0.0);
        wmin = fabs(w) < wmin ? fabs(w) : wmin;
        wmax = dmax(wmax, fabs(w));
        blk[dev::block_at(np, i, 0)] = (float)((double)P[4 * i + 0] - w * cx);
        blk[dev::block_at(np, i, 1)] = (float)((double)P[4 * i + 1] - w * cy);
        blk[dev::block_at(np, i, 2)] = (float)((double)P[4 * i + 2] - w * cz);
        blk[dev::block_at(np, i, 3)] = (float)w;
        if (w != 0.0) {
            const double dx = P[4 * i] / w - cx, dy = P[4 * i + 1] / w - cy, dz = P[4 * i + 2] / w - cz;
            rad = dmax(rad, sqrt(dx * dx + dy * dy + dz * dz));
        }
    }
    for (int i = n; i < np; ++i) {  // padding, never read as a point
        blk[dev::block_at(np, i, 0)] = 0.f; blk[dev::block_at(np, i, 1)] = 0.f; blk[dev::block_at(np, i, 2)] = 0.f;
        blk[dev::block_at(np, i, 3)] = 1.f;
    }
    const int flags = (pos ? dev::kFlagPositiveWeights : 0) | (wmax > dev::kWideWeightRatio * wmin ? dev::kFlagWideWeights : 0);
    hdr = make_int4((int)off, p | (q << 4) | (flags << 8), patch_id, surf);
    ctr = make_double4(cx, cy, cz, rad);
    const int ci[4] = {0, p * (q + 1), p * (q + 1) + q, q};  // q00, q10, q11, q01 (bezier_patch.h:37-44)
    for (int c = 0; c < 4; ++c) {
        const float* X = P + 4 * ci[c];
        const float iw = 1.f / X[3];
        corners[c] = make_float4(X[0] * iw, X[1] * iw, X[2] * iw, 0.f);
    }
    delta = patch_delta(P, p, q);
    frame = patch_frame(P, p, q, cx, cy, cz, b);
    patch_obb(P, p, q, obb);
}

}  // namespace nrt
