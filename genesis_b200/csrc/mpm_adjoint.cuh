// Reverse-mode adjoint of one MPM substep for Elastic (corotated) particles with
// per-particle Lame parameters.  Included by mpm_kernels.cu (same module, namespace gbm).
//
// Forward being differentiated (reference: mpm_solver.py:261-449, elastic.py:70-75,
// legacy_coupler.py:364-375, 495-496):
//   F_tmp = (I + dt C) F;  F_tmp = U S V^T;  R = U V^T;  J = det F_tmp
//   P = 2 mu (F_tmp - R) F_tmp^T + lam J (J - 1) I;   A = s P + m C
//   m_i = sum w m;  p_i = sum w (m v + A d_i)                     (d_i = x_i - x_p)
//   v_i = bc(p_i / m_i + dt g)
//   v' = sum w v_i;  C' = c sum w v_i u_i^T;  x' = clamp(x + dt v'), v'' = bc(v')
//                                                                (u_i = d_i / dx, c = 4 inv_dx)
// Three kernels run after the forward grid of the substep has been recomputed:
//   k_adj_g2p   particles: adjoint of the gather; scatters the grid-velocity adjoint
//   k_adj_grid  nodes:     adjoint of p/m + dt g and the boundary
//   k_adj_p2g   particles: adjoint of the scatter, the stress (polar rotation via the
//               closed-form SVD adjoint U [(M_ij - M_ji)/(s_i + s_j)] V^T), J, F_tmp
// The adjoint arrays use the state's planar layout (channel c of slot s at c*stride + s).
#pragma once

struct AdjWs {
    float* state;      // scratch copy of the state for the forward recompute
    float4* saved_mm;  // momentum.xyz + mass of the recomputed p2g
    float4* vbar;      // adjoint of the grid velocity (xyz)
    float4* pmbar;     // adjoint of momentum (xyz) and mass (w)
    float* xbar;       // [3][stride] x adjoint from the g2p part
    int64_t stride;
};

static inline uint64_t adj_layout(const mpm_problem& p, uint64_t* off /*5*/) {
    const uint64_t n = (uint64_t)p.n_particles;
    const uint64_t stride = align_up(n > 0 ? n : 1, 64);
    const uint64_t nodes = (uint64_t)p.n_blocks * BLK3;
    const uint64_t sizes[5] = {stride * MPM_STATE_CH * 4, nodes * 16, nodes * 16, nodes * 16, stride * 3 * 4};
    uint64_t o = 0;
    for (int i = 0; i < 5; ++i) {
        off[i] = o;
        o = align_up(o + sizes[i], 256);
    }
    return o;
}

static inline AdjWs adj_ws_of(const mpm_problem& p, void* base) {
    uint64_t off[5];
    adj_layout(p, off);
    char* b = (char*)base;
    AdjWs a;
    a.state = (float*)(b + off[0]);
    a.saved_mm = (float4*)(b + off[1]);
    a.vbar = (float4*)(b + off[2]);
    a.pmbar = (float4*)(b + off[3]);
    a.xbar = (float*)(b + off[4]);
    a.stride = (int64_t)align_up(p.n_particles > 0 ? p.n_particles : 1, 64);
    return a;
}

__device__ __forceinline__ float& w_vbar_x(const AdjWs& a, int64_t n) { return a.vbar[n].x; }
__device__ __forceinline__ float& w_vbar_y(const AdjWs& a, int64_t n) { return a.vbar[n].y; }
__device__ __forceinline__ float& w_vbar_z(const AdjWs& a, int64_t n) { return a.vbar[n].z; }

__device__ __forceinline__ void bspline_d(float fx, float* w, float* dw) {
    const float a = 1.5f - fx, b = fx - 1.f, c = fx - 0.5f;
    w[0] = 0.5f * a * a;
    w[1] = 0.75f - b * b;
    w[2] = 0.5f * c * c;
    dw[0] = -a;
    dw[1] = -2.f * b;
    dw[2] = c;
}

__device__ __forceinline__ bool node_ok(const mpm_instance& I, int gx, int gy, int gz) {
    return gx >= 0 && gy >= 0 && gz >= 0 && gx < I.res[0] && gy < I.res[1] && gz < I.res[2];
}

// ---- adjoint of g2p (mpm_solver.py:396-437)
__global__ void k_adj_g2p(mpm_problem prob, const mpm_instance* __restrict__ inst, mpm_particles par, float* adj,
                          Ws w, AdjWs aw) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= prob.n_particles || !(par.pflags[s] & MPM_PFLAG_ACTIVE)) return;
    const mpm_instance& I = inst[find_instance_by_particle(inst, prob.n_instances, s)];
    const int64_t st = par.state_stride;
    float x[3], fx[3], wv[3][3], dwv[3][3];
    int base[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) x[d] = par.state[(MPM_CH_X + d) * st + s];
    if (!finite3(x[0], x[1], x[2])) return;
    locate(I, x, base, fx);
#pragma unroll
    for (int d = 0; d < 3; ++d) bspline_d(fx[d], wv[d], dwv[d]);
    // recompute the gathered velocity for the boundary masks
    float nv[3] = {0.f, 0.f, 0.f};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k) {
                const int gx = base[0] + i, gy = base[1] + j, gz = base[2] + k;
                if (!node_ok(I, gx, gy, gz)) continue;
                const float4 g = w.gv[node_addr(I, gx, gy, gz)];
                const float wt = wv[0][i] * wv[1][j] * wv[2][k];
                nv[0] += wt * g.x;
                nv[1] += wt * g.y;
                nv[2] += wt * g.z;
            }
    float gxb[3], vb[3], Cb[9];
    const float* xin = adj + (int64_t)MPM_CH_X * st;
    const float* vin = adj + (int64_t)MPM_CH_V * st;
    const float* cin = adj + (int64_t)MPM_CH_C * st;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const float xs = x[d] + I.dt * nv[d];
        const bool clamped = xs > I.bnd_hi[d] || xs < I.bnd_lo[d];
        const bool vzero = (xs >= I.bnd_hi[d] && nv[d] >= 0.f) || (xs <= I.bnd_lo[d] && nv[d] <= 0.f);
        gxb[d] = clamped ? 0.f : xin[d * st + s];
        vb[d] = (vzero ? 0.f : vin[d * st + s]) + I.dt * gxb[d];
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) Cb[k] = cin[k * st + s];
    float xb[3] = {gxb[0], gxb[1], gxb[2]};
    const float c = I.c_scale;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k) {
                const int gx = base[0] + i, gy = base[1] + j, gz = base[2] + k;
                if (!node_ok(I, gx, gy, gz)) continue;
                const int64_t na = node_addr(I, gx, gy, gz);
                const float4 g = w.gv[na];
                const float vh[3] = {g.x, g.y, g.z};
                const float wt = wv[0][i] * wv[1][j] * wv[2][k];
                const float gw[3] = {dwv[0][i] * wv[1][j] * wv[2][k] * I.inv_dx, wv[0][i] * dwv[1][j] * wv[2][k] * I.inv_dx,
                                     wv[0][i] * wv[1][j] * dwv[2][k] * I.inv_dx};
                const float u[3] = {(float)i - fx[0], (float)j - fx[1], (float)k - fx[2]};
                float Cu[3];
#pragma unroll
                for (int a = 0; a < 3; ++a) Cu[a] = Cb[a * 3 + 0] * u[0] + Cb[a * 3 + 1] * u[1] + Cb[a * 3 + 2] * u[2];
                atomicAdd(&w_vbar_x(aw, na), wt * vb[0] + c * wt * Cu[0]);
                atomicAdd(&w_vbar_y(aw, na), wt * vb[1] + c * wt * Cu[1]);
                atomicAdd(&w_vbar_z(aw, na), wt * vb[2] + c * wt * Cu[2]);
                const float wbar = vb[0] * vh[0] + vb[1] * vh[1] + vb[2] * vh[2] +
                                   c * (vh[0] * Cu[0] + vh[1] * Cu[1] + vh[2] * Cu[2]);
#pragma unroll
                for (int e = 0; e < 3; ++e) {
                    const float ub = c * wt * (Cb[0 * 3 + e] * vh[0] + Cb[1 * 3 + e] * vh[1] + Cb[2 * 3 + e] * vh[2]);
                    xb[e] += wbar * gw[e] - I.inv_dx * ub;
                }
            }
#pragma unroll
    for (int d = 0; d < 3; ++d) aw.xbar[d * aw.stride + s] = xb[d];
}

// ---- adjoint of the grid update (legacy_coupler.py:364-375, 495-496)
__global__ void k_adj_grid(mpm_problem prob, const mpm_instance* __restrict__ inst, Ws w, AdjWs aw) {
    const int64_t node = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (node >= prob.n_blocks * BLK3) return;
    const int64_t blk = node / BLK3;
    const int ln = (int)(node % BLK3);
    const mpm_instance& I = inst[find_instance_by_block(inst, prob.n_instances, blk)];
    const float4 mm = aw.saved_mm[node];
    float4 out = make_float4(0.f, 0.f, 0.f, 0.f);
    if (mm.w > I.eps) {
        const BlockCoord bc = block_coord((int)(blk - I.blk_base), I);
        const int lxyz[3] = {ln / (BLK * BLK), (ln / BLK) % BLK, ln % BLK};
        const int bxyz[3] = {bc.bx, bc.by, bc.bz};
        const float inv = 1.f / mm.w;
        const float pm[3] = {mm.x, mm.y, mm.z};
        const float4 vb4 = aw.vbar[node];
        const float vbin[3] = {vb4.x, vb4.y, vb4.z};
        float vb[3], dotp = 0.f;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const float v = inv * pm[d] + I.dt * I.gravity[d];
            const float pos = (float)(bxyz[d] * BLK + lxyz[d] + I.lower_cell[d]) * I.dx;
            const bool zero = (pos >= I.bnd_hi[d] && v >= 0.f) || (pos <= I.bnd_lo[d] && v <= 0.f);
            vb[d] = zero ? 0.f : vbin[d];
            dotp += vb[d] * pm[d];
        }
        out = make_float4(vb[0] * inv, vb[1] * inv, vb[2] * inv, -dotp * inv * inv);
    }
    aw.pmbar[node] = out;
}

// cofactor matrix of F (= det(F) F^-T)
__device__ __forceinline__ void cofactor(const float* F, float* K) {
    K[0] = F[4] * F[8] - F[5] * F[7];
    K[1] = F[5] * F[6] - F[3] * F[8];
    K[2] = F[3] * F[7] - F[4] * F[6];
    K[3] = F[2] * F[7] - F[1] * F[8];
    K[4] = F[0] * F[8] - F[2] * F[6];
    K[5] = F[1] * F[6] - F[0] * F[7];
    K[6] = F[1] * F[5] - F[2] * F[4];
    K[7] = F[2] * F[3] - F[0] * F[5];
    K[8] = F[0] * F[4] - F[1] * F[3];
}

// ---- adjoint of p2g, the corotated stress and compute_F_tmp (mpm_solver.py:261-389)
__global__ void k_adj_p2g(mpm_problem prob, const mpm_instance* __restrict__ inst,
                          const mpm_material* __restrict__ mats, mpm_particles par, float* adj, float* lame_bar,
                          AdjWs aw) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= prob.n_particles || !(par.pflags[s] & MPM_PFLAG_ACTIVE)) return;
    const mpm_instance& I = inst[find_instance_by_particle(inst, prob.n_instances, s)];
    const mpm_material m = mats[I.mat_base + par.mat[s]];
    const int64_t st = par.state_stride;
    const float* S = par.state;
    float x[3], v[3], C[9], F[9];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        x[d] = S[(MPM_CH_X + d) * st + s];
        v[d] = S[(MPM_CH_V + d) * st + s];
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        C[k] = S[(MPM_CH_C + k) * st + s];
        F[k] = S[(MPM_CH_F + k) * st + s];
    }
    if (!finite3(x[0], x[1], x[2])) return;
    const float mu = par.mu_p ? par.mu_p[s] : m.mu;
    const float lam = par.lam_p ? par.lam_p[s] : m.lam;
    // forward recompute
    float Ft[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            float acc = F[i * 3 + j];
#pragma unroll
            for (int k = 0; k < 3; ++k) acc += I.dt * C[i * 3 + k] * F[k * 3 + j];
            Ft[i * 3 + j] = acc;
        }
    float U[9], Sg[3], V[9], Rm[9];
    svd3(Ft, U, Sg, V);
    uvt(U, V, Rm);
    const float J = Sg[0] * (Sg[1] * Sg[2]);
    const bool neo = (m.flags & MPM_MATF_NEOHOOKEAN) != 0;
    // muscle actuation (muscle.py:57-65): + ka g g^T with g = F_tmp d, ka = stiffness * actu
    const bool musc = (m.flags & MPM_MATF_MUSCLE) && par.actu;
    float dd[3] = {0.f, 0.f, 0.f}, g[3] = {0.f, 0.f, 0.f}, ka = 0.f;
    if (musc) {
        const int gi = par.gid[s];
#pragma unroll
        for (int a = 0; a < 3; ++a) dd[a] = par.muscle_dir[3 * gi + a];
        ka = m.muscle_stiffness * par.actu[gi];
#pragma unroll
        for (int a = 0; a < 3; ++a) g[a] = Ft[a * 3 + 0] * dd[0] + Ft[a * 3 + 1] * dd[1] + Ft[a * 3 + 2] * dd[2];
    }
    float P[9];
    if (neo) {
        // mu F_tmp F_tmp^T + (lam log J - mu) I   (elastic.py:78-81)
        const float dg = lam * logf(J) - mu;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
                P[i * 3 + j] = mu * (Ft[i * 3 + 0] * Ft[j * 3 + 0] + Ft[i * 3 + 1] * Ft[j * 3 + 1] +
                                     Ft[i * 3 + 2] * Ft[j * 3 + 2]) + (i == j ? dg : 0.f);
    } else {
        corotated(mu, lam, J, Ft, Rm, P);
    }
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) P[i * 3 + j] += ka * g[i] * g[j];
    const float mass = m.mass;
    float A[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) A[k] = I.stress_scale * P[k] + mass * C[k];
    float fx[3], wv[3][3], dwv[3][3];
    int base[3];
    locate(I, x, base, fx);
#pragma unroll
    for (int d = 0; d < 3; ++d) bspline_d(fx[d], wv[d], dwv[d]);
    // adjoint of the scatter
    float xb[3] = {aw.xbar[0 * aw.stride + s], aw.xbar[1 * aw.stride + s], aw.xbar[2 * aw.stride + s]};
    float vbn[3] = {0.f, 0.f, 0.f};
    float Ab[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    const float dx = I.dx;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k) {
                const int gx = base[0] + i, gy = base[1] + j, gz = base[2] + k;
                if (!node_ok(I, gx, gy, gz)) continue;
                const float4 pmb = aw.pmbar[node_addr(I, gx, gy, gz)];
                const float pb[3] = {pmb.x, pmb.y, pmb.z};
                const float wt = wv[0][i] * wv[1][j] * wv[2][k];
                const float gw[3] = {dwv[0][i] * wv[1][j] * wv[2][k] * I.inv_dx, wv[0][i] * dwv[1][j] * wv[2][k] * I.inv_dx,
                                     wv[0][i] * wv[1][j] * dwv[2][k] * I.inv_dx};
                const float d[3] = {((float)i - fx[0]) * dx, ((float)j - fx[1]) * dx, ((float)k - fx[2]) * dx};
                float wbar = pmb.w * mass;
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    const float q = mass * v[a] + A[a * 3 + 0] * d[0] + A[a * 3 + 1] * d[1] + A[a * 3 + 2] * d[2];
                    wbar += pb[a] * q;
                    vbn[a] += wt * mass * pb[a];
#pragma unroll
                    for (int b = 0; b < 3; ++b) Ab[a * 3 + b] += wt * pb[a] * d[b];
                }
#pragma unroll
                for (int e = 0; e < 3; ++e)
                    xb[e] += wbar * gw[e] - wt * (A[0 * 3 + e] * pb[0] + A[1 * 3 + e] * pb[1] + A[2 * 3 + e] * pb[2]);
            }
    // A = s P + m C
    float Pb[9], Cbn[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        Pb[k] = I.stress_scale * Ab[k];
        Cbn[k] = mass * Ab[k];
    }
    float Ftb[9];
    float mub = 0.f, lamb = 0.f;
    if (musc) {
        // P += ka g g^T: gb = ka (Pb + Pb^T) g, Ftb += gb d^T, dL/dactu = stiffness g^T Pb g
        float gb[3], gPg = 0.f;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            gb[a] = 0.f;
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                gb[a] += ka * (Pb[a * 3 + b] + Pb[b * 3 + a]) * g[b];
                gPg += g[a] * Pb[a * 3 + b] * g[b];
            }
        }
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) Ftb[a * 3 + b] = gb[a] * dd[b];
        lame_bar[2 * st + s] += m.muscle_stiffness * gPg;
    } else {
#pragma unroll
        for (int k = 0; k < 9; ++k) Ftb[k] = 0.f;
    }
    if (neo) {
        // P = mu F F^T + (lam log J - mu) I: Ftb += mu (Pb + Pb^T) F + lam tr(Pb) / J dJ/dF
        const float trP = Pb[0] + Pb[4] + Pb[8];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                float acc = 0.f;
#pragma unroll
                for (int k = 0; k < 3; ++k) acc += (Pb[i * 3 + k] + Pb[k * 3 + i]) * Ft[k * 3 + j];
                Ftb[i * 3 + j] += mu * acc;
                mub += Pb[i * 3 + j] * (Ft[i * 3 + 0] * Ft[j * 3 + 0] + Ft[i * 3 + 1] * Ft[j * 3 + 1] +
                                        Ft[i * 3 + 2] * Ft[j * 3 + 2]);
            }
        mub -= trP;
        lamb = trP * logf(J);
        float K[9];
        cofactor(Ft, K);
        const float Jb = lam * trP / J;
#pragma unroll
        for (int k = 0; k < 9; ++k) Ftb[k] += Jb * K[k];
    } else {
    // P = 2 mu (Ft - R) Ft^T + lam J (J - 1) I
    float D[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) D[k] = Ft[k] - Rm[k];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const float dft = D[i * 3 + 0] * Ft[j * 3 + 0] + D[i * 3 + 1] * Ft[j * 3 + 1] + D[i * 3 + 2] * Ft[j * 3 + 2];
            mub += Pb[i * 3 + j] * dft;
        }
    mub *= 2.f;
    const float trP = Pb[0] + Pb[4] + Pb[8];
    lamb = trP * J * (J - 1.f);
    float Rb[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            float a1 = 0.f, a2 = 0.f, a3 = 0.f;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                a1 += Pb[i * 3 + k] * Ft[k * 3 + j];  // (Pb Ft)_ij
                a2 += Pb[k * 3 + i] * D[k * 3 + j];   // (Pb^T D)_ij
            }
            a3 = a1;
            Ftb[i * 3 + j] += 2.f * mu * (a1 + a2);
            Rb[i * 3 + j] = -2.f * mu * a3;
        }
    const float Jb = lam * (2.f * J - 1.f) * trP;
    float K[9];
    cofactor(Ft, K);
#pragma unroll
    for (int k = 0; k < 9; ++k) Ftb[k] += Jb * K[k];
    // polar rotation: Ftb += U X V^T, X_ij = (M_ij - M_ji) / (s_i + s_j), M = U^T Rb V
    float T[9], M[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            T[i * 3 + j] = Rb[i * 3 + 0] * V[0 * 3 + j] + Rb[i * 3 + 1] * V[1 * 3 + j] + Rb[i * 3 + 2] * V[2 * 3 + j];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            M[i * 3 + j] = U[0 * 3 + i] * T[0 * 3 + j] + U[1 * 3 + i] * T[1 * 3 + j] + U[2 * 3 + i] * T[2 * 3 + j];
    float X[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const float den = Sg[i] + Sg[j];
            X[i * 3 + j] = (i == j || fabsf(den) < 1e-12f) ? 0.f : (M[i * 3 + j] - M[j * 3 + i]) / den;
        }
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            float acc = 0.f;
#pragma unroll
            for (int a = 0; a < 3; ++a)
#pragma unroll
                for (int b = 0; b < 3; ++b) acc += U[i * 3 + a] * X[a * 3 + b] * V[j * 3 + b];
            Ftb[i * 3 + j] += acc;
        }
    }
    // F_new = F_tmp (Elastic): the incoming F adjoint adds to F_tmp's
    float* xo = adj + (int64_t)MPM_CH_X * st;
    float* vo = adj + (int64_t)MPM_CH_V * st;
    float* co = adj + (int64_t)MPM_CH_C * st;
    float* fo = adj + (int64_t)MPM_CH_F * st;
#pragma unroll
    for (int k = 0; k < 9; ++k) Ftb[k] += fo[k * st + s];
    // F_tmp = (I + dt C) F
    float Fbn[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            float a = Ftb[i * 3 + j];  // identity part
            float cb = 0.f;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                a += I.dt * C[k * 3 + i] * Ftb[k * 3 + j];  // ((dt C)^T Ftb)_ij
                cb += Ftb[i * 3 + k] * F[j * 3 + k];        // (Ftb F^T)_ij
            }
            Fbn[i * 3 + j] = a;
            Cbn[i * 3 + j] += I.dt * cb;
        }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        xo[d * st + s] = xb[d];
        vo[d * st + s] = vbn[d];
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        co[k * st + s] = Cbn[k];
        fo[k * st + s] = Fbn[k];
    }
    lame_bar[s] += mub;
    lame_bar[st + s] += lamb;
}
