// Per-material return mapping and stress for the fused p2g kernel.
//
// Each branch restates one gs.materials.MPM class:
//   Elastic        materials/MPM/elastic.py:62-83
//   ElastoPlastic  materials/MPM/elasto_plastic.py:66-93 (stress: base.py:83-90)
//   Liquid         materials/MPM/liquid.py:50-64
//   Sand           materials/MPM/sand.py:51-89
//   Snow           materials/MPM/snow.py:62-81
// and the call protocol of p2g (mpm_solver.py:303-345): J is det(S) of F_tmp's SVD,
// Snow's hardening uses the previous Jp, Sand's stress uses S_new, Liquid's uses F_tmp.
#pragma once

#include "../../include/genesis_b200_mpm.h"

namespace gbm {

// M = U diag(s) V^T
__device__ __forceinline__ void usvt(const float* U, const float* s, const float* V, float* M) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            M[i * 3 + j] = U[i * 3 + 0] * s[0] * V[j * 3 + 0] + U[i * 3 + 1] * s[1] * V[j * 3 + 1] +
                           U[i * 3 + 2] * s[2] * V[j * 3 + 2];
}

// R = U V^T
__device__ __forceinline__ void uvt(const float* U, const float* V, float* R) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            R[i * 3 + j] = U[i * 3 + 0] * V[j * 3 + 0] + U[i * 3 + 1] * V[j * 3 + 1] + U[i * 3 + 2] * V[j * 3 + 2];
}

// out = U diag(d) U^T + c I (symmetric: six entries computed)
__device__ __forceinline__ void udut(const float* U, const float* d, float c, float* out) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = i; j < 3; ++j) {
            const float acc = U[i * 3 + 0] * d[0] * U[j * 3 + 0] + U[i * 3 + 1] * d[1] * U[j * 3 + 1] +
                              U[i * 3 + 2] * d[2] * U[j * 3 + 2];
            out[i * 3 + j] = acc + (i == j ? c : 0.f);
            out[j * 3 + i] = out[i * 3 + j];
        }
}

// The corotated stress of F_new = U diag(sn) V^T in the SVD basis (the return-mapped
// materials build F_new so): 2 mu (F_new - U V^T) F_new^T = U diag(2 mu (sn - 1) sn) U^T, so
// out = U diag(2 mu (sn - 1) sn) U^T + lam J (J - 1) I.  Besides ~50 fewer instructions than
// the matrix form, it takes sn - 1 from sn itself rather than from the difference of two
// reconstructed matrices (float32 cancellation at the small strains of a yield surface).
__device__ __forceinline__ void corotated_svd(float mu, float lam, float J, const float* U, const float* sn,
                                              float* out) {
    const float d[3] = {2.f * mu * (sn[0] - 1.f) * sn[0], 2.f * mu * (sn[1] - 1.f) * sn[1],
                        2.f * mu * (sn[2] - 1.f) * sn[2]};
    udut(U, d, lam * J * (J - 1.f), out);
}

// out = 2 mu (F - R) F^T + lam J (J - 1) I   (corotated form, base.py:86-88)
__device__ __forceinline__ void corotated(float mu, float lam, float J, const float* F, const float* R, float* out) {
    const float two_mu = 2.f * mu;
    const float diag = lam * J * (J - 1.f);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            float acc = (F[i * 3 + 0] - R[i * 3 + 0]) * F[j * 3 + 0] + (F[i * 3 + 1] - R[i * 3 + 1]) * F[j * 3 + 1] +
                        (F[i * 3 + 2] - R[i * 3 + 2]) * F[j * 3 + 2];
            out[i * 3 + j] = two_mu * acc + (i == j ? diag : 0.f);
        }
}

// Logarithms, exponentials and quotients of the return mappings: CUDA's logf / expf and IEEE
// division (about 1 ulp of the result).  GBM_FAST_MATH=1 selects the MUFU-based forms
// instead (absolute error ~1e-7 in log near 1, relative ~1e-7 in exp, 2 ulp in the quotient),
// as the reference's fast_math build does: measured 0.5% faster per substep on the 500k mixed
// scene, within the same parity tolerances; the accurate forms are the default.
#ifndef GBM_FAST_MATH
#define GBM_FAST_MATH 0
#endif
__device__ __forceinline__ float flog(float x) { return GBM_FAST_MATH ? __logf(x) : logf(x); }
__device__ __forceinline__ float fexp(float x) { return GBM_FAST_MATH ? __expf(x) : expf(x); }
__device__ __forceinline__ float fdiv(float a, float b) { return GBM_FAST_MATH ? __fdividef(a, b) : a / b; }

// Inviscid Liquid needs only J from the SVD (its stress is lam J (J - 1) I).
__device__ __forceinline__ bool needs_uv(const mpm_material& m, float mu) {
    return !(m.kind == MPM_MAT_LIQUID && mu == 0.f);
}

// Return mapping + stress for one particle.
//   in : material m (mu/lam possibly overridden per particle), eps = gs.EPS,
//        J = det(S), F_tmp, U, S, V, Jp (previous frame)
//   out: F_new, Jp_new, stress (unscaled Kirchhoff-type stress of update_stress)
__device__ __forceinline__ void constitutive(const mpm_material& m, float mu, float lam, float eps, float J,
                                             const float* Ft, const float* U, const float* S, const float* V,
                                             float Jp, float* F_new, float& Jp_new, float* stress) {
    float R[9];
    switch (m.kind) {
        case MPM_MAT_ELASTIC: {
#pragma unroll
            for (int k = 0; k < 9; ++k) F_new[k] = Ft[k];
            Jp_new = Jp;
            if (m.flags & MPM_MATF_NEOHOOKEAN) {
                // mu F_tmp F_tmp^T + (lam log J - mu) I   (elastic.py:78-81)
                const float d = lam * flog(J) - mu;
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int j = 0; j < 3; ++j) {
                        float acc = Ft[i * 3 + 0] * Ft[j * 3 + 0] + Ft[i * 3 + 1] * Ft[j * 3 + 1] + Ft[i * 3 + 2] * Ft[j * 3 + 2];
                        stress[i * 3 + j] = mu * acc + (i == j ? d : 0.f);
                    }
            } else {
                uvt(U, V, R);
                corotated(mu, lam, J, F_new, R, stress);
            }
            break;
        }
        case MPM_MAT_LIQUID: {
            // F_new = J^(1/3) I (liquid.py:52); pow(J, 1/3) is NaN for a negative J
            const float c = J >= 0.f ? cbrtf(J) : __int_as_float(0x7fc00000);
#pragma unroll
            for (int k = 0; k < 9; ++k) F_new[k] = (k % 4 == 0) ? c : 0.f;
            Jp_new = Jp;
            if (mu == 0.f) {
                // liquid.py:47-48: mu is 0 unless viscous, so 2 mu (F_tmp - R) F_tmp^T vanishes
                const float diag = lam * J * (J - 1.f);
#pragma unroll
                for (int k = 0; k < 9; ++k) stress[k] = (k % 4 == 0) ? diag : 0.f;
            } else {
                uvt(U, V, R);
                corotated(mu, lam, J, Ft, R, stress);  // liquid.py:60 uses F_tmp
            }
            break;
        }
        case MPM_MAT_ELASTOPLASTIC: {
            float Sn[3];
            if (m.flags & MPM_MATF_VON_MISES) {
                // elasto_plastic.py:71-84
                float e[3];
#pragma unroll
                for (int d = 0; d < 3; ++d) e[d] = flog(fmaxf(S[d], 0.05f));
                const float mean = (e[0] + e[1] + e[2]) * (1.f / 3.f);
                float eh[3] = {e[0] - mean, e[1] - mean, e[2] - mean};
                const float ehn = sqrtf(eh[0] * eh[0] + eh[1] * eh[1] + eh[2] * eh[2] + eps);
                const float dg = ehn - m.vm_threshold * (m.mu / mu);
                if (dg > 0.f) {
                    const float r = fdiv(dg, ehn);
#pragma unroll
                    for (int d = 0; d < 3; ++d) Sn[d] = fexp(e[d] - r * eh[d]);
                    usvt(U, Sn, V, F_new);
                } else {
#pragma unroll
                    for (int k = 0; k < 9; ++k) F_new[k] = Ft[k];
#pragma unroll
                    for (int d = 0; d < 3; ++d) Sn[d] = S[d];
                }
            } else {
#pragma unroll
                for (int d = 0; d < 3; ++d) Sn[d] = fminf(fmaxf(S[d], m.clamp_lo), m.clamp_hi);
                usvt(U, Sn, V, F_new);
            }
            Jp_new = Jp;
            corotated_svd(mu, lam, J, U, Sn, stress);
            break;
        }
        case MPM_MAT_SNOW: {
            float Sn[3];
            float jp = Jp;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                Sn[d] = fminf(fmaxf(S[d], m.clamp_lo), m.clamp_hi);
                jp = jp * fdiv(S[d], Sn[d]);
            }
            Jp_new = jp;
            usvt(U, Sn, V, F_new);
            // snow.py:75-79: hardening from the previous Jp
            const float h = fexp(10.f * (1.f - Jp));
            corotated_svd(mu * h, lam * h, J, U, Sn, stress);
            break;
        }
        case MPM_MAT_SAND:
        default: {
            // sand.py:52-77
            // ls = log S_new: S_new = exp(ls) is built from its logarithm, so sand.py:82's
            // log(S_new) is ls itself (0 when the return mapping projects to the tip)
            float e[3], Sn[3], ls[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) e[d] = flog(fmaxf(fabsf(S[d]), 1e-4f));
            const float tr = e[0] + e[1] + e[2] + Jp;
            const float t3 = tr * (1.f / 3.f);
            float eh[3] = {e[0] - t3, e[1] - t3, e[2] - t3};
            const float ehn = sqrtf(eh[0] * eh[0] + eh[1] * eh[1] + eh[2] * eh[2] + eps);
            if (tr >= 0.f) {
                Jp_new = tr;
                Sn[0] = Sn[1] = Sn[2] = 1.f;
                ls[0] = ls[1] = ls[2] = 0.f;
            } else {
                Jp_new = 0.f;
                const float c1 = fdiv(3.f * lam + 2.f * mu, 2.f * mu);
                const float dg = ehn + c1 * tr * m.sand_alpha;
                const float r = fdiv(fmaxf(0.f, dg), ehn);
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    ls[d] = e[d] - r * eh[d];
                    Sn[d] = fexp(ls[d]);
                }
            }
            usvt(U, Sn, V, F_new);
            // sand.py:80-88 with S = S_new: U diag(center) V^T F_new^T with center_i =
            // (2 mu ls_i + lam sum ls) / S_new_i and F_new = U diag(S_new) V^T, i.e.
            // U diag(2 mu ls_i + lam sum ls) U^T
            const float lsum = ls[0] + ls[1] + ls[2];
            const float d[3] = {2.f * mu * ls[0] + lam * lsum, 2.f * mu * ls[1] + lam * lsum,
                                2.f * mu * ls[2] + lam * lsum};
            udut(U, d, 0.f, stress);
            break;
        }
    }
}

}  // namespace gbm
