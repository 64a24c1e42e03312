// Register-resident 3x3 singular value decomposition for the p2g kernel.
//
// Replaces ti.svd(F_tmp) at genesis/engine/solvers/mpm_solver.py:273.  gstaichi's
// ti.svd follows McAdams et al. 2011 ("Computing the Singular Value Decomposition of
// 3x3 matrices with minimal branching and elementary floating point operations"),
// whose structure this implementation keeps:
//   1. cyclic Jacobi eigen-analysis of the symmetric A^T A, accumulating V as a
//      product of plane rotations (so det V = +1),
//   2. sort the columns of B = A V by decreasing squared norm, negating one column on
//      every swap so V stays a proper rotation,
//   3. QR of B with non-negative r00 and r11, giving a proper rotation U and the
//      singular values on the diagonal of R; only the last one can be negative
//      (det A < 0).  The paper's Givens rotations are replaced by Gram-Schmidt on the first
//      two columns and a cross product for the third (the same factorisation: the QR with
//      r00, r11 >= 0 is unique for rank >= 2), about 40 fewer instructions per particle
//      (the fused kernel measured 1.2% faster per substep).
// Unlike the paper's quaternion "approximate Givens" rotations, the Jacobi step uses
// exact rotations (Golub & Van Loan, Alg. 8.4.2) with at most 4 sweeps: 4 cyclic sweeps
// leave relative off-diagonal residue below 1e-20 for F = I + E with |E| up to 0.5
// (3 sweeps: ~6e-6), i.e. float32 round-off; a warp stops earlier, between two rotations,
// once all its lanes have converged to that level (typically after 7-8 rotations).
#pragma once

namespace gbm {

// unroll factor of the Jacobi sweep loop (1: rolled, smaller code; 4: fully unrolled)
#ifndef GBM_SVD_UNROLL
#define GBM_SVD_UNROLL 1
#endif
constexpr int kSvdUnroll = GBM_SVD_UNROLL;
// early-exit level of the Jacobi sweeps: off-diagonal mass of A^T A against its trace
#ifndef GBM_SVD_TOL
#define GBM_SVD_TOL 1e-7f
#endif

// One Jacobi rotation in plane (P, Q) of the symmetric matrix a, accumulated into v.
template <int P, int Q>
__device__ __forceinline__ void jacobi_pq(float (&a)[3][3], float (&v)[3][3]) {
    constexpr int R = 3 - P - Q;
    const float apq = a[P][Q];
    const float app = a[P][P];
    const float aqq = a[Q][Q];
    // The smaller root of t^2 + 2 tau t - 1 = 0 (tau = (aqq - app) / (2 apq)), written without
    // tau: with d = aqq - app and e = 2 apq, t = sign(d) e / (|d| + sqrt(d^2 + e^2)), so
    // |t| <= 1 and one reciprocal and two reciprocal square roots make the rotation.
    // Approximate reciprocal / rsqrt: the rotation only needs to be orthogonal to round-off,
    // which c = rsqrt(1 + t^2), s = t c guarantees whatever t is.  Branch-free; an apq too
    // small for e^2 to stay a normal float selects the identity rotation t = 0.
    const float d = aqq - app;
    const float e = 2.f * apq;
    const float r2 = fmaf(d, d, e * e);
    const float den = fabsf(d) + r2 * rsqrtf(fmaxf(r2, 1e-37f));
    float t = __fdividef(e, copysignf(den, d));
    t = (fabsf(apq) > 1e-18f) ? t : 0.f;
    const float c = rsqrtf(1.f + t * t);
    const float s = t * c;
    a[P][P] = app - t * apq;
    a[Q][Q] = aqq + t * apq;
    a[P][Q] = 0.f;
    a[Q][P] = 0.f;
    const float arp = a[R][P];
    const float arq = a[R][Q];
    const float nrp = c * arp - s * arq;
    const float nrq = s * arp + c * arq;
    a[R][P] = nrp;
    a[P][R] = nrp;
    a[R][Q] = nrq;
    a[Q][R] = nrq;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float vip = v[i][P];
        const float viq = v[i][Q];
        v[i][P] = c * vip - s * viq;
        v[i][Q] = s * vip + c * viq;
    }
}

// One-sided Jacobi rotation of columns (P, Q) of B = A V (and of V) that makes them
// orthogonal.  The 2x2 Gram entries are dot products of B's own columns, accurate relative
// to |b_P| |b_Q|, so this resolves directions that the eigen-analysis of A^T A (accurate
// only relative to |A|^2) cannot: the small singular directions of an ill-conditioned A.
template <int P, int Q>
__device__ __forceinline__ void onesided_pq(float (&b)[3][3], float (&v)[3][3]) {
    const float app = b[0][P] * b[0][P] + b[1][P] * b[1][P] + b[2][P] * b[2][P];
    const float aqq = b[0][Q] * b[0][Q] + b[1][Q] * b[1][Q] + b[2][Q] * b[2][Q];
    const float apq = b[0][P] * b[0][Q] + b[1][P] * b[1][Q] + b[2][P] * b[2][Q];
    const float d = aqq - app;
    const float e = 2.f * apq;
    const float r2 = fmaf(d, d, e * e);
    const float den = fabsf(d) + r2 * rsqrtf(fmaxf(r2, 1e-37f));
    float t = __fdividef(e, copysignf(den, d));
    t = (fabsf(apq) > 1e-30f) ? t : 0.f;
    const float c = rsqrtf(1.f + t * t);
    const float s = t * c;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float bp = b[i][P], bq = b[i][Q];
        b[i][P] = c * bp - s * bq;
        b[i][Q] = s * bp + c * bq;
        const float vp = v[i][P], vq = v[i][Q];
        v[i][P] = c * vp - s * vq;
        v[i][Q] = s * vp + c * vq;
    }
}

template <int I, int J>
__device__ __forceinline__ void swap_cols_neg(float (&b)[3][3], float (&v)[3][3], float& ni, float& nj) {
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        float tb = b[r][I];
        b[r][I] = b[r][J];
        b[r][J] = -tb;
        float tv = v[r][I];
        v[r][I] = v[r][J];
        v[r][J] = -tv;
    }
    float tn = ni;
    ni = nj;
    nj = tn;
}

// A (row-major, 9 floats) = U diag(S) V^T with U, V proper rotations (row-major).
// need_uv = false: the caller uses only the product S0 S1 S2 (= det A, which the QR
// below yields whatever V is), so this lane does not hold up the warp's Jacobi sweeps.
template <int SWEEPS = 4>
__device__ __forceinline__ void svd3(const float* A, float* U, float* S, float* V, bool need_uv = true) {
    float a[3][3];
    // A^T A
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = i; j < 3; ++j) {
            float acc = A[0 * 3 + i] * A[0 * 3 + j] + A[1 * 3 + i] * A[1 * 3 + j] + A[2 * 3 + i] * A[2 * 3 + j];
            a[i][j] = acc;
            a[j][i] = acc;
        }
    float v[3][3] = {{1.f, 0.f, 0.f}, {0.f, 1.f, 0.f}, {0.f, 0.f, 1.f}};
    // Early exit, decided per warp before every rotation: once every active lane's
    // off-diagonal mass is below 1e-7 of its diagonal, a further rotation moves the diagonal
    // by O(1e-14) and V by O(1e-7), i.e. float32 round-off (and when eigenvalues nearly
    // coincide, a rotation inside that eigenspace leaves U S V^T, and every isotropic function
    // of F, unchanged).  The diagonal sum is the trace, which the rotations keep, so the
    // threshold is fixed up front.  Checking before each rotation rather than each sweep
    // saves 1.3-1.7 of the ~8.8 rotations a warp of the plastic materials makes.  (A tighter
    // threshold, or one relative to each pair's own diagonal, changes neither the benchmark
    // scenes' trajectories nor the small-direction accuracy below, measured: the limit there
    // is forming A^T A in float32, which the one-sided sweep after the QR ordering addresses.)
    const float thr = GBM_SVD_TOL * (a[0][0] + a[1][1] + a[2][2]);
    auto converged = [&]() {
        return __all_sync(__activemask(), !need_uv || !(fabsf(a[0][1]) + fabsf(a[0][2]) + fabsf(a[1][2]) > thr));
    };
#pragma unroll kSvdUnroll
    for (int sw = 0; sw < SWEEPS; ++sw) {
        if (converged()) break;
        jacobi_pq<0, 1>(a, v);
        if (converged()) break;
        jacobi_pq<0, 2>(a, v);
        if (converged()) break;
        jacobi_pq<1, 2>(a, v);
    }
    // B = A V
    float b[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            b[i][j] = A[i * 3 + 0] * v[0][j] + A[i * 3 + 1] * v[1][j] + A[i * 3 + 2] * v[2][j];
    float n0 = b[0][0] * b[0][0] + b[1][0] * b[1][0] + b[2][0] * b[2][0];
    float n1 = b[0][1] * b[0][1] + b[1][1] * b[1][1] + b[2][1] * b[2][1];
    float n2 = b[0][2] * b[0][2] + b[1][2] * b[1][2] + b[2][2] * b[2][2];
    // Ill-conditioned A (a singular value below 1e-2 of the largest): V from A^T A is
    // accurate only to ~1e-7 |A|^2 / gap in the small directions; one one-sided sweep on the
    // columns of B restores relative accuracy.  Decided per warp, so well-conditioned warps
    // (all of them in ordinary scenes) skip it.
    {
        const float nmax = fmaxf(n0, fmaxf(n1, n2)), nmin = fminf(n0, fminf(n1, n2));
        if (__any_sync(__activemask(), need_uv && nmin < 1e-4f * nmax)) {
            onesided_pq<0, 1>(b, v);
            onesided_pq<0, 2>(b, v);
            onesided_pq<1, 2>(b, v);
            n0 = b[0][0] * b[0][0] + b[1][0] * b[1][0] + b[2][0] * b[2][0];
            n1 = b[0][1] * b[0][1] + b[1][1] * b[1][1] + b[2][1] * b[2][1];
            n2 = b[0][2] * b[0][2] + b[1][2] * b[1][2] + b[2][2] * b[2][2];
        }
    }
    if (n0 < n1) swap_cols_neg<0, 1>(b, v, n0, n1);
    if (n0 < n2) swap_cols_neg<0, 2>(b, v, n0, n2);
    if (n1 < n2) swap_cols_neg<1, 2>(b, v, n1, n2);
    // QR of B by Gram-Schmidt: u0 = b0 / |b0|, u1 = the part of b1 orthogonal to u0,
    // normalised, u2 = u0 x u1 (so det U = +1), R's diagonal (|b0|, |b1 - (u0.b1) u0|, u2.b2).
    // This is the QR with r00, r11 >= 0 (unique for rank >= 2).  A (near) zero b0 selects u0 = e_x; a b1 parallel to u0 selects for u1 the
    // unit vector orthogonal to u0 in the plane of u0 and the axis u0 is least aligned with.
    {
        const bool ok0 = n0 > 1e-30f;
        const float r0 = rsqrtf(ok0 ? n0 : 1.f);
        const float u0[3] = {ok0 ? b[0][0] * r0 : 1.f, ok0 ? b[1][0] * r0 : 0.f, ok0 ? b[2][0] * r0 : 0.f};
        const float d01 = u0[0] * b[0][1] + u0[1] * b[1][1] + u0[2] * b[2][1];
        float w1[3] = {b[0][1] - d01 * u0[0], b[1][1] - d01 * u0[1], b[2][1] - d01 * u0[2]};
        float m1 = w1[0] * w1[0] + w1[1] * w1[1] + w1[2] * w1[2];
        if (!(m1 > 1e-30f)) {
            // rank <= 1: e_k - (u0.e_k) u0 for the k of the smallest |u0_k|
            const float a0 = fabsf(u0[0]), a1 = fabsf(u0[1]), a2 = fabsf(u0[2]);
            const int k = (a0 <= a1 && a0 <= a2) ? 0 : (a1 <= a2 ? 1 : 2);
            const float uk = k == 0 ? u0[0] : (k == 1 ? u0[1] : u0[2]);
            w1[0] = (k == 0 ? 1.f : 0.f) - uk * u0[0];
            w1[1] = (k == 1 ? 1.f : 0.f) - uk * u0[1];
            w1[2] = (k == 2 ? 1.f : 0.f) - uk * u0[2];
            m1 = w1[0] * w1[0] + w1[1] * w1[1] + w1[2] * w1[2];
        }
        const float r1 = rsqrtf(m1);
        const float u1[3] = {w1[0] * r1, w1[1] * r1, w1[2] * r1};
        const float u2[3] = {u0[1] * u1[2] - u0[2] * u1[1], u0[2] * u1[0] - u0[0] * u1[2],
                             u0[0] * u1[1] - u0[1] * u1[0]};
        S[0] = ok0 ? n0 * r0 : 0.f;
        S[1] = u1[0] * b[0][1] + u1[1] * b[1][1] + u1[2] * b[2][1];
        S[2] = u2[0] * b[0][2] + u2[1] * b[1][2] + u2[2] * b[2][2];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            U[i * 3 + 0] = u0[i];
            U[i * 3 + 1] = u1[i];
            U[i * 3 + 2] = u2[i];
#pragma unroll
            for (int j = 0; j < 3; ++j) V[i * 3 + j] = v[i][j];
        }
    }
}

}  // namespace gbm
