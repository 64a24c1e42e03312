// Reverse-mode adjoint of one MPM substep for every MPM material (Elastic corotated /
// neo-Hookean, Muscle, ElastoPlastic von Mises / clamp, Liquid, Sand, Snow) with
// per-particle Lame parameters.  Included by mpm_kernels.cu (same module, namespace gbm).
//
// Forward being differentiated (reference: mpm_solver.py:261-449, materials/MPM/*.py,
// legacy_coupler.py:364-375, 495-496):
//   F_tmp = (I + dt C) F;  F_tmp = U S V^T;  J = det S
//   (F_new, Jp_new) = the material's return mapping; P = its stress
//   A = s P + m C;  m_i = sum w m;  p_i = sum w (m v + A d_i)          (d_i = x_i - x_p)
//   v_i = bc(p_i / m_i + dt g)
//   v' = sum w v_i;  C' = c sum w v_i u_i^T;  x' = clamp(x + dt v'), v'' = bc(v')
//                                                                (u_i = d_i / dx, c = 4 inv_dx)
// Three kernels run after the forward grid of the substep has been recomputed:
//   k_adj_g2p   particles: adjoint of the gather; scatters the grid-velocity adjoint
//   k_adj_grid  nodes:     adjoint of p/m + dt g and the boundary
//   k_adj_p2g   particles: adjoint of the scatter, the material (material_adjoint: the return
//               mapping, the stress and the SVD together, in the SVD basis), J, F_tmp
// The adjoint arrays use the state's planar layout (channel c of slot s at c*stride + s),
// the Jp channel included (Snow and Sand carry Jp from one substep to the next).
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
    // recompute the gathered velocity for the boundary masks.  The 27 node velocities are
    // loaded once, all issued before the first is used (one CTA per SM at the differentiable
    // scenes' sizes: the loads' latency, not bandwidth, sets this kernel's time), and kept in
    // registers for the scatter below.
    float4 gn[27];
#pragma unroll
    for (int n = 0; n < 27; ++n) {
        const int gx = base[0] + n / 9, gy = base[1] + (n / 3) % 3, gz = base[2] + n % 3;
        gn[n] = node_ok(I, gx, gy, gz) ? w.gv[node_addr(I, gx, gy, gz)] : make_float4(0.f, 0.f, 0.f, 0.f);
    }
    float nv[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int n = 0; n < 27; ++n) {
        const float wt = wv[0][n / 9] * wv[1][(n / 3) % 3] * wv[2][n % 3];
        nv[0] += wt * gn[n].x;
        nv[1] += wt * gn[n].y;
        nv[2] += wt * gn[n].z;
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
#pragma unroll
    for (int n = 0; n < 27; ++n) {
        const int i = n / 9, j = (n / 3) % 3, k = n % 3;
        const int gx = base[0] + i, gy = base[1] + j, gz = base[2] + k;
        if (!node_ok(I, gx, gy, gz)) continue;
        const int64_t na = node_addr(I, gx, gy, gz);
        const float vh[3] = {gn[n].x, gn[n].y, gn[n].z};
        const float wt = wv[0][i] * wv[1][j] * wv[2][k];
        const float gw[3] = {dwv[0][i] * wv[1][j] * wv[2][k] * I.inv_dx, wv[0][i] * dwv[1][j] * wv[2][k] * I.inv_dx,
                             wv[0][i] * wv[1][j] * dwv[2][k] * I.inv_dx};
        const float u[3] = {(float)i - fx[0], (float)j - fx[1], (float)k - fx[2]};
        float Cu[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) Cu[a] = Cb[a * 3 + 0] * u[0] + Cb[a * 3 + 1] * u[1] + Cb[a * 3 + 2] * u[2];
        // one 16-byte vector reduction per node (sm_90+) instead of three scalar ones
        atomicAdd(&aw.vbar[na], make_float4(wt * vb[0] + c * wt * Cu[0], wt * vb[1] + c * wt * Cu[1],
                                            wt * vb[2] + c * wt * Cu[2], 0.f));
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
// ---- adjoint of the colliders' responses (legacy_coupler.py:297-350, tool_entity/mesh.py:147-176)

// Adjoint of the shared response v' = vc + (rt sc - n rn e) infl + rv (1 - infl) with rv = v - vc,
// rn = rv.n (acting only where rn < 0), rt = rv - rn n, sc = max(0, |rt|_eps + rn mu) / |rt|_eps
// (|x|_eps = sqrt(|x|^2 + eps), e the restitution): given ob = dL/dv', returns dL/drv, dL/dn and
// dL/dinfl (dL/dvc = ob - dL/drv).
__device__ __forceinline__ void respond_vjp(const float* rv, const float* n, float infl, float mu, float e, float eps,
                                            const float* ob, float* rvb, float* nb, float& inflb) {
    const float rn = rv[0] * n[0] + rv[1] * n[1] + rv[2] * n[2];
    const float rt[3] = {rv[0] - rn * n[0], rv[1] - rn * n[1], rv[2] - rn * n[2]};
    const float rtn = sqrtf(rt[0] * rt[0] + rt[1] * rt[1] + rt[2] * rt[2] + eps);
    const float m = rtn + rn * mu;
    const float mp = fmaxf(0.f, m);
    const float sc = mp / rtn;
    float rtb[3], scb = 0.f, rnb = 0.f;
    inflb = 0.f;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float rnew = rt[i] * sc - n[i] * rn * e;
        inflb += ob[i] * (rnew - rv[i]);
        const float rnewb = ob[i] * infl;
        rvb[i] = ob[i] * (1.f - infl);
        rtb[i] = rnewb * sc;
        scb += rnewb * rt[i];
        rnb -= e * rnewb * n[i];
        nb[i] = -e * rnewb * rn;
    }
    float rtnb = -scb * mp / (rtn * rtn);
    if (m > 0.f) {
        const float mb = scb / rtn;
        rtnb += mb;
        rnb += mb * mu;
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        rtb[i] += rtnb * rt[i] / rtn;
        rvb[i] += rtb[i];
    }
    rnb -= rtb[0] * n[0] + rtb[1] * n[1] + rtb[2] * n[2];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        nb[i] -= rn * rtb[i];
        rvb[i] += rnb * n[i];
        nb[i] += rnb * rv[i];
    }
}

// The trilinear voxel sample of tool_sdf_at and its gradient with respect to the voxel
// coordinate (d(1 - |d|)/dpv = -1 for d >= 0, +1 below); zero gradient outside the grid,
// where the sample is the constant 1.
__device__ __forceinline__ float tool_sdf_grad_at(const float* __restrict__ vox, int res, const float* pv, float* g) {
    g[0] = g[1] = g[2] = 0.f;
    const float f0 = floorf(pv[0]), f1 = floorf(pv[1]), f2 = floorf(pv[2]);
    if (!(f0 >= 0.f && f1 >= 0.f && f2 >= 0.f && f0 < (float)(res - 1) && f1 < (float)(res - 1) &&
          f2 < (float)(res - 1)))
        return 1.f;
    const int b0 = (int)f0, b1 = (int)f1, b2 = (int)f2;
    float sd = 0.f;
#pragma unroll
    for (int o = 0; o < 8; ++o) {
        const int i = o >> 2, j = (o >> 1) & 1, k = o & 1;
        const float d0 = pv[0] - (float)(b0 + i), d1 = pv[1] - (float)(b1 + j), d2 = pv[2] - (float)(b2 + k);
        const float a0 = 1.f - fabsf(d0), a1 = 1.f - fabsf(d1), a2 = 1.f - fabsf(d2);
        const float val = vox[((int64_t)(b0 + i) * res + (b1 + j)) * res + (b2 + k)];
        sd += a0 * a1 * a2 * val;
        g[0] += (d0 >= 0.f ? -1.f : 1.f) * a1 * a2 * val;
        g[1] += (d1 >= 0.f ? -1.f : 1.f) * a0 * a2 * val;
        g[2] += (d2 >= 0.f ? -1.f : 1.f) * a0 * a1 * val;
    }
    return sd;
}

// Adjoint of collide_tool at grid node p with input velocity v: vb holds dL/d(output velocity)
// on entry and dL/dv on return; dL/d(tool position) and dL/d(tool linear velocity) are added
// to pb and lb.  The influence, the normal (central differences of the trilinear sample, so
// its derivative is the difference of the sample's gradients) and the body point's velocity
// all depend on the tool's position; the rotation is taken as given.
__device__ void collide_tool_vjp(const mpm_collider& c, const float* __restrict__ sdf_voxels, float eps, float dt,
                                 const float* p, const float* v, float* vb, float* pb, float* lb) {
    if (!sdf_voxels || c.sdf_res < 2) return;
    const float* vox = sdf_voxels + c.sdf_offset;
    const int res = c.sdf_res;
    const float q[3] = {p[0] - c.pos[0], p[1] - c.pos[1], p[2] - c.pos[2]};
    const float half = 0.5f * (float)(res - 1);
    float pv[3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
        pv[i] = c.sdf_scale[i] * (c.rot[0 * 3 + i] * q[0] + c.rot[1 * 3 + i] * q[1] + c.rot[2 * 3 + i] * q[2]) + half;
    float gsd[3];
    const float sd = tool_sdf_grad_at(vox, res, pv, gsd);
    const float soft = fmaxf(eps, c.softness);
    const float ex = expf(-sd / soft);
    const float infl = fminf(ex, 1.f);
    if (!(sd <= 0.f || infl > 0.1f)) return;
    // vel_collider: ((E - I) q + dpos) / dt, (E - I) q = M q with M = sin(th) K + 2 sin^2(th / 2) K^2
    float M[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    {
        const float wx = c.ang_vel[0] * dt, wy = c.ang_vel[1] * dt, wz = c.ang_vel[2] * dt;
        const float th = sqrtf(wx * wx + wy * wy + wz * wz);
        if (th > 0.f) {
            const float k[3] = {wx / th, wy / th, wz / th};
            const float K[9] = {0.f, -k[2], k[1], k[2], 0.f, -k[0], -k[1], k[0], 0.f};
            const float sh = sinf(0.5f * th), s = sinf(th), t = 2.f * sh * sh;
#pragma unroll
            for (int a = 0; a < 3; ++a)
#pragma unroll
                for (int b = 0; b < 3; ++b)
                    M[a * 3 + b] = s * K[a * 3 + b] + t * (K[a * 3 + 0] * K[0 * 3 + b] + K[a * 3 + 1] * K[1 * 3 + b] +
                                                           K[a * 3 + 2] * K[2 * 3 + b]);
        }
    }
    float dz = c.lin_vel[2] * dt;
    const bool clamped = c.pos[2] + dz < c.floor;
    if (clamped) dz = c.floor - c.pos[2];
    float vc[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) vc[i] = (M[i * 3 + 0] * q[0] + M[i * 3 + 1] * q[1] + M[i * 3 + 2] * q[2]) / dt;
    vc[0] += c.lin_vel[0];
    vc[1] += c.lin_vel[1];
    vc[2] += dz / dt;
    const float rv[3] = {v[0] - vc[0], v[1] - vc[1], v[2] - vc[2]};
    // the normal and the Jacobian H of its central differences: H_ij = d nv_i / d pv_j
    float nv[3], H[9];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        float a[3] = {pv[0], pv[1], pv[2]}, b[3] = {pv[0], pv[1], pv[2]};
        a[i] += 1e-2f;
        b[i] -= 1e-2f;
        float ga[3], gb[3];
        nv[i] = (tool_sdf_grad_at(vox, res, a, ga) - tool_sdf_grad_at(vox, res, b, gb)) / 2e-2f;
#pragma unroll
        for (int j = 0; j < 3; ++j) H[i * 3 + j] = (ga[j] - gb[j]) / 2e-2f;
    }
    const float s1 = rsqrtf(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2] + eps);
    const float nm[3] = {nv[0] * s1 / c.sdf_scale[0], nv[1] * s1 / c.sdf_scale[1], nv[2] * s1 / c.sdf_scale[2]};
    float nr[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) nr[i] = c.rot[i * 3 + 0] * nm[0] + c.rot[i * 3 + 1] * nm[1] + c.rot[i * 3 + 2] * nm[2];
    const float s2 = rsqrtf(nr[0] * nr[0] + nr[1] * nr[1] + nr[2] * nr[2] + eps);
    const float n[3] = {nr[0] * s2, nr[1] * s2, nr[2] * s2};
    const float rn = rv[0] * n[0] + rv[1] * n[1] + rv[2] * n[2];
    if (!(rn < 0.f)) return;
    const float ob[3] = {vb[0], vb[1], vb[2]};
    float rvb[3], nb[3], inflb;
    respond_vjp(rv, n, infl, c.friction, 0.f, eps, ob, rvb, nb, inflb);
    const float vcb[3] = {ob[0] - rvb[0], ob[1] - rvb[1], ob[2] - rvb[2]};
    // n = nr s2 -> nr; nr = R nm -> nm; nm = nv s1 / scale -> nv
    const float dn = nr[0] * nb[0] + nr[1] * nb[1] + nr[2] * nb[2];
    float nrb[3], nmb[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) nrb[i] = s2 * nb[i] - s2 * s2 * s2 * nr[i] * dn;
#pragma unroll
    for (int i = 0; i < 3; ++i)
        nmb[i] = (c.rot[0 * 3 + i] * nrb[0] + c.rot[1 * 3 + i] * nrb[1] + c.rot[2 * 3 + i] * nrb[2]) / c.sdf_scale[i];
    const float dv = nv[0] * nmb[0] + nv[1] * nmb[1] + nv[2] * nmb[2];
    float nvb[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) nvb[i] = s1 * nmb[i] - s1 * s1 * s1 * nv[i] * dv;
    // pv: the normal's differences and the influence
    const float sdb = (ex < 1.f) ? -inflb * infl / soft : 0.f;
    float pvb[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) pvb[j] = H[0 * 3 + j] * nvb[0] + H[1 * 3 + j] * nvb[1] + H[2 * 3 + j] * nvb[2] + sdb * gsd[j];
    // pv = scale (R^T q) + half, and vc's rotation part M q / dt
    float qb[3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
        qb[i] = c.rot[i * 3 + 0] * c.sdf_scale[0] * pvb[0] + c.rot[i * 3 + 1] * c.sdf_scale[1] * pvb[1] +
                c.rot[i * 3 + 2] * c.sdf_scale[2] * pvb[2] +
                (M[0 * 3 + i] * vcb[0] + M[1 * 3 + i] * vcb[1] + M[2 * 3 + i] * vcb[2]) / dt;
    // q = p - pos; vc's translation: lin_vel, or (floor - pos_z) / dt once clamped
    pb[0] -= qb[0];
    pb[1] -= qb[1];
    pb[2] -= qb[2];
    lb[0] += vcb[0];
    lb[1] += vcb[1];
    if (clamped)
        pb[2] -= vcb[2] / dt;
    else
        lb[2] += vcb[2];
#pragma unroll
    for (int i = 0; i < 3; ++i) vb[i] = rvb[i];
}

// Adjoint of collide_rigid with respect to the node velocity only (the geom's pose and
// velocity are taken as given): vb holds dL/d(output velocity) on entry, dL/dv on return.
__device__ void collide_rigid_vjp(const mpm_collider& c, const float* __restrict__ sdf, float eps, const float* p,
                                  const float* v, float* vb) {
    float sd, g[3], q[3], n[3];
    sdf_grad(c, sdf, eps, p, sd, g, q);
    const float infl = fminf(expf(-sd / fmaxf(1e-10f, c.softness)), 1.f);
    if (!(infl > 0.1f)) return;
    unit_normal(c, eps, g, n);
    const float vr[3] = {c.lin_vel[0] + c.ang_vel[1] * q[2] - c.ang_vel[2] * q[1],
                         c.lin_vel[1] + c.ang_vel[2] * q[0] - c.ang_vel[0] * q[2],
                         c.lin_vel[2] + c.ang_vel[0] * q[1] - c.ang_vel[1] * q[0]};
    const float rv[3] = {v[0] - vr[0], v[1] - vr[1], v[2] - vr[2]};
    if (!(rv[0] * n[0] + rv[1] * n[1] + rv[2] * n[2] < 0.f)) return;
    const float ob[3] = {vb[0], vb[1], vb[2]};
    float nb[3], inflb;
    respond_vjp(rv, n, infl, c.friction, c.restitution, eps, ob, vb, nb, inflb);
}

// The grid op's collider chain on one node, stopped before collider `stop` of the given kind
// (tools first in index order, then the rigid geoms): the velocity that collider receives.
__device__ void collider_chain(const mpm_collider* __restrict__ cs, int nc, int inst, const float* __restrict__ sdf,
                               float eps, float dt, const float* p, float* v, bool stop_tool, int stop) {
    for (int k = 0; k < nc; ++k) {
        if (cs[k].instance != inst || cs[k].kind != MPM_COLLIDER_TOOL) continue;
        if (stop_tool && k == stop) return;
        collide_tool(cs[k], sdf, eps, dt, p, v);
    }
    for (int k = 0; k < nc; ++k) {
        if (cs[k].instance != inst || cs[k].kind == MPM_COLLIDER_TOOL) continue;
        if (!stop_tool && k == stop) return;
        collide_rigid(cs[k], sdf, eps, dt, 0.f, p, v, nullptr);
    }
}

__device__ __forceinline__ float warp_sum(float x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

// Adjoint of one force field's v += acc(p, v) dt with respect to v (its Jacobian is symmetric):
// vb holds dL/d(v after) on entry and dL/d(v before) on return.  CONSTANT, WIND and
// TURBULENCE's noise do not depend on v; NOISE is refused by differentiable scenes.
__device__ void force_field_vjp(const mpm_force_field& f, float eps, float dt, const float* p, const float* v,
                                float* vb) {
    switch (f.kind) {
        case MPM_FF_POINT: {
            const float c = 1.f - dt * f.flow * point_falloff(f, eps, p);
            vb[0] *= c;
            vb[1] *= c;
            vb[2] *= c;
            break;
        }
        case MPM_FF_DRAG: {
            const float vn = sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
            const float dot = v[0] * vb[0] + v[1] * vb[1] + v[2] * vb[2];
            const float q = vn > 0.f ? dt * f.quadratic * dot / vn : 0.f;
            const float c = 1.f - dt * (f.linear + f.quadratic * vn);
#pragma unroll
            for (int d = 0; d < 3; ++d) vb[d] = c * vb[d] - q * v[d];
            break;
        }
        case MPM_FF_VORTEX: {
            const float c = 1.f - dt * f.damping;
            vb[0] *= c;
            vb[1] *= c;
            vb[2] *= c;
            break;
        }
        case MPM_FF_TURBULENCE: {
            const float c = 1.f - dt * f.flow;
            vb[0] *= c;
            vb[1] *= c;
            vb[2] *= c;
            break;
        }
        default:
            break;
    }
}

// Adjoint of the grid op per node: the boundary, the colliders' responses in reverse order
// (tools' position / linear-velocity adjoints summed per warp into cbar[6 k ..]), the force
// fields in reverse order, then v = p / m + dt g.  Every thread runs the collider loops, so
// the warp sums see full warps.
__global__ void k_adj_grid(mpm_problem prob, const mpm_instance* __restrict__ inst, Ws w, AdjWs aw,
                           const mpm_collider* __restrict__ cs, int nc, const float* __restrict__ sdf, float* cbar,
                           const mpm_force_field* __restrict__ ffs, int n_ff, const int* __restrict__ ff_perm) {
    const int64_t node = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = node < prob.n_blocks * BLK3;
    const int64_t blk = in ? node / BLK3 : 0;
    const int ln = (int)(node % BLK3);
    const int ii = in ? find_instance_by_block(inst, prob.n_instances, blk) : 0;
    const mpm_instance& I = inst[ii];
    const float4 mm = in ? aw.saved_mm[node] : make_float4(0.f, 0.f, 0.f, 0.f);
    const bool act = in && mm.w > I.eps;
    float4 out = make_float4(0.f, 0.f, 0.f, 0.f);
    float p[3] = {0.f, 0.f, 0.f}, vin[3] = {0.f, 0.f, 0.f}, vb[3] = {0.f, 0.f, 0.f}, pm[3] = {mm.x, mm.y, mm.z};
    const float inv = act ? 1.f / mm.w : 0.f;
    if (act) {
        const BlockCoord bc = block_coord((int)(blk - I.blk_base), I);
        const int lxyz[3] = {ln / (BLK * BLK), (ln / BLK) % BLK, ln % BLK};
        const int bxyz[3] = {bc.bx, bc.by, bc.bz};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            vin[d] = inv * pm[d] + I.dt * I.gravity[d];
            p[d] = (float)(bxyz[d] * BLK + lxyz[d] + I.lower_cell[d]) * I.dx;
        }
        if (n_ff > 0) apply_force_fields(ffs, n_ff, ff_perm, I.eps, I.dt, p, vin, node, 0u);
        float v[3] = {vin[0], vin[1], vin[2]};  // vin: the colliders' input from here on
        if (nc > 0) collider_chain(cs, nc, ii, sdf, I.eps, I.dt, p, v, false, nc);
        const float4 vb4 = aw.vbar[node];
        const float vbin[3] = {vb4.x, vb4.y, vb4.z};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const bool zero = (p[d] >= I.bnd_hi[d] && v[d] >= 0.f) || (p[d] <= I.bnd_lo[d] && v[d] <= 0.f);
            vb[d] = zero ? 0.f : vbin[d];
        }
    }
    // the colliders in reverse order: the rigid geoms, then the tools
    for (int pass = 0; pass < 2; ++pass) {
        const bool tools = pass == 1;
        for (int k = nc - 1; k >= 0; --k) {
            const bool is_tool = cs[k].kind == MPM_COLLIDER_TOOL;
            if (is_tool != tools) continue;
            float pb[3] = {0.f, 0.f, 0.f}, lb[3] = {0.f, 0.f, 0.f};
            if (act && cs[k].instance == ii) {
                float vk[3] = {vin[0], vin[1], vin[2]};
                collider_chain(cs, nc, ii, sdf, I.eps, I.dt, p, vk, tools, k);
                if (tools)
                    collide_tool_vjp(cs[k], sdf, I.eps, I.dt, p, vk, vb, pb, lb);
                else
                    collide_rigid_vjp(cs[k], sdf, I.eps, p, vk, vb);
            }
            if (tools && cbar) {
                float r[6] = {pb[0], pb[1], pb[2], lb[0], lb[1], lb[2]};
#pragma unroll
                for (int j = 0; j < 6; ++j) {
                    r[j] = warp_sum(r[j]);
                    if ((threadIdx.x & 31) == 0 && r[j] != 0.f) atomicAdd(&cbar[6 * k + j], r[j]);
                }
            }
        }
    }
    if (act && n_ff > 0) {
        // the force fields in reverse order, each from the velocity it received
        for (int k = n_ff - 1; k >= 0; --k) {
            if (!ffs[k].active) continue;
            float vk[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) vk[d] = inv * pm[d] + I.dt * I.gravity[d];
            apply_force_fields(ffs, k, ff_perm, I.eps, I.dt, p, vk, node, 0u);
            force_field_vjp(ffs[k], I.eps, I.dt, p, vk, vb);
        }
    }
    if (act) {
        const float dotp = vb[0] * pm[0] + vb[1] * pm[1] + vb[2] * pm[2];
        out = make_float4(vb[0] * inv, vb[1] * inv, vb[2] * inv, -dotp * inv * inv);
    }
    if (in) aw.pmbar[node] = out;
}

// The grid op's adjoint over the active blocks a recorded substep lists (no colliders: the
// recorded reverse pass refuses them), with the same per-node arithmetic as k_adj_grid.
// vbar is cleared behind the read, so it is zero again for the substep before (whose g2p
// adjoint writes only inside its own active blocks) without a pass over the whole grid.
__global__ void __launch_bounds__(256) k_adj_grid_active(mpm_problem prob, const mpm_instance* __restrict__ inst,
                                                         AdjWs aw, const int2* __restrict__ active,
                                                         const uint32_t* __restrict__ n_active_p,
                                                         const mpm_force_field* __restrict__ ffs, int n_ff,
                                                         const int* __restrict__ ff_perm) {
    const int n_active = (int)*n_active_p;
    const int gpc = blockDim.x / BLK3;
    const int grp = threadIdx.x / BLK3;
    const int ln = threadIdx.x % BLK3;
    const int lxyz[3] = {ln / (BLK * BLK), (ln / BLK) % BLK, ln % BLK};
    for (int i = blockIdx.x * gpc + grp; i < n_active; i += gridDim.x * gpc) {
        const int2 e = active[i];
        const mpm_instance& I = inst[e.x];
        const BlockCoord bc = unpack_bc(e.y);
        const int64_t node = (I.blk_base + local_block(I, bc.bx, bc.by, bc.bz)) * BLK3 + ln;
        const float4 mm = aw.saved_mm[node];
        const bool act = mm.w > I.eps;
        float4 out = make_float4(0.f, 0.f, 0.f, 0.f);
        if (act) {
            const float inv = 1.f / mm.w;
            const float pm[3] = {mm.x, mm.y, mm.z};
            const int bxyz[3] = {bc.bx, bc.by, bc.bz};
            float p[3], v[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                v[d] = inv * pm[d] + I.dt * I.gravity[d];
                p[d] = (float)(bxyz[d] * BLK + lxyz[d] + I.lower_cell[d]) * I.dx;
            }
            if (n_ff > 0) apply_force_fields(ffs, n_ff, ff_perm, I.eps, I.dt, p, v, node, 0u);
            const float4 vb4 = aw.vbar[node];
            const float vbin[3] = {vb4.x, vb4.y, vb4.z};
            float vb[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const bool zero = (p[d] >= I.bnd_hi[d] && v[d] >= 0.f) || (p[d] <= I.bnd_lo[d] && v[d] <= 0.f);
                vb[d] = zero ? 0.f : vbin[d];
            }
            // the force fields in reverse order, each from the velocity it received
            for (int k = n_ff - 1; k >= 0; --k) {
                if (!ffs[k].active) continue;
                float vk[3];
#pragma unroll
                for (int d = 0; d < 3; ++d) vk[d] = inv * pm[d] + I.dt * I.gravity[d];
                apply_force_fields(ffs, k, ff_perm, I.eps, I.dt, p, vk, node, 0u);
                force_field_vjp(ffs[k], I.eps, I.dt, p, vk, vb);
            }
            const float dotp = vb[0] * pm[0] + vb[1] * pm[1] + vb[2] * pm[2];
            out = make_float4(vb[0] * inv, vb[1] * inv, vb[2] * inv, -dotp * inv * inv);
        }
        aw.pmbar[node] = out;
        aw.vbar[node] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
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

// ---- the materials' adjoint in the SVD basis
// Every material's F_new is U diag(g(s)) V^T (Liquid: J^(1/3) I) and its stress
// U diag(p(s)) U^T (plus the Muscle term, handled by the caller), with g and p symmetric
// functions of the singular values s of F_tmp.  Their adjoint follows from g, p, their
// Jacobians and divided differences:
//   X = U^T Fn_bar V,  Z = U^T sym(P_bar) U
//   s_bar_k = sum_i X_ii dg_i/ds_k + Z_ii dp_i/ds_k + Jpn_bar dJp_new/ds_k
//   Y_ij = 1/2 [(X_ij + X_ji) (g_i - g_j)/(s_i - s_j) + (X_ij - X_ji) (g_i + g_j)/(s_i + s_j)]
//          + 2 Z_ij s_j (p_i - p_j) / (s_i^2 - s_j^2)                         (i != j)
//   F_tmp_bar += U (diag(s_bar) + Y) V^T
// This is the reference's backward (gstaichi autodiff of update_F_S_Jp / update_stress
// with U, S, V as inputs, then backward_svd, mpm_solver.py:1112-1129) rearranged: equal to it
// wherever its signmax(s_j^2 - s_i^2, 1e-6) guard is inactive, and the derivative that guard
// approximates where it is not.  The divided differences are formed through
// log(c_i / c_j) = log1p((c_i - c_j) / c_j) and expm1, so they stay exact as s_i -> s_j (the
// rest state and every small strain).

// (g_i - g_j) / (s_i - s_j) where g_i - g_j = g_j expm1(kappa log(c_i / c_j)) and c is the
// clamped |s| (c = |s| where unclamped); its limit at s_i = s_j is g_j kappa / s_j (0 if clamped)
__device__ __forceinline__ float ddiff_log(float si, float sj, float ci, float cj, float kappa, float gj) {
    const float den = si - sj;
    if (den != 0.f) return gj * expm1f(kappa * log1pf((ci - cj) / cj)) / den;
    return ci == fabsf(si) ? gj * kappa / sj : 0.f;
}

struct Spec {
    float g[3], p[3];
    float Dg[3][3], Dp[3][3];    // dg_i/ds_k, dp_i/ds_k
    float DDg[3][3], DDp[3][3];  // (g_i - g_j)/(s_i - s_j), (p_i - p_j)/(s_i - s_j)
    float dg_dJp[3], dp_dJp[3], dg_dmu[3], dp_dmu[3], dg_dlam[3], dp_dlam[3];
    float dJpn_ds[3], dJpn_dJp;
    bool ident;   // F_new = F_tmp
    bool liquid;  // F_new = J^(1/3) I
};

// p_i = 2 muc (g_i - 1) g_i + lamc J (J - 1) (the corotated stress's eigenvalues, base.py:86-88)
__device__ __forceinline__ void spec_corot(Spec& o, float muc, float lamc, float J, const float* Jk) {
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        o.p[i] = 2.f * muc * (o.g[i] - 1.f) * o.g[i] + lamc * J * (J - 1.f);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            o.Dp[i][k] = 2.f * muc * (2.f * o.g[i] - 1.f) * o.Dg[i][k] + lamc * (2.f * J - 1.f) * Jk[k];
            o.DDp[i][k] = 2.f * muc * (o.g[i] + o.g[k] - 1.f) * o.DDg[i][k];
        }
        o.dp_dmu[i] = 2.f * (o.g[i] - 1.f) * o.g[i] + 2.f * muc * (2.f * o.g[i] - 1.f) * o.dg_dmu[i];
        o.dp_dlam[i] = J * (J - 1.f);
    }
}

__device__ __forceinline__ void spec_ident(Spec& o, const float* s) {
    o.ident = true;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        o.g[i] = s[i];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            o.Dg[i][k] = i == k ? 1.f : 0.f;
            o.DDg[i][k] = 1.f;
        }
    }
}

// g, p and their derivatives for one material (materials/MPM/*.py, as p2g calls them)
__device__ void material_spectral(const mpm_material& m, float mu, float lam, float eps, const float* s, float Jp,
                                  Spec& o) {
    const float Jk[3] = {s[1] * s[2], s[0] * s[2], s[0] * s[1]};
    const float J = s[0] * Jk[0];
    o.ident = o.liquid = false;
    o.dJpn_dJp = 1.f;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        o.dg_dJp[i] = o.dp_dJp[i] = o.dg_dmu[i] = o.dg_dlam[i] = o.dJpn_ds[i] = 0.f;
#pragma unroll
        for (int k = 0; k < 3; ++k) o.Dg[i][k] = o.DDg[i][k] = 0.f;
    }
    switch (m.kind) {
        case MPM_MAT_ELASTIC:
            spec_ident(o, s);
            if (m.flags & MPM_MATF_NEOHOOKEAN) {  // p_i = mu s_i^2 + lam log J - mu (elastic.py:78-81)
                const float lj = logf(J);
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    o.p[i] = mu * s[i] * s[i] + lam * lj - mu;
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        o.Dp[i][k] = (i == k ? 2.f * mu * s[i] : 0.f) + lam * Jk[k] / J;
                        o.DDp[i][k] = mu * (s[i] + s[k]);
                    }
                    o.dp_dmu[i] = s[i] * s[i] - 1.f;
                    o.dp_dlam[i] = lj;
                }
            } else {
                spec_corot(o, mu, lam, J, Jk);
            }
            break;
        case MPM_MAT_LIQUID:  // F_new = J^(1/3) I; stress corotated on F_tmp (liquid.py:50-64)
            spec_ident(o, s);
            o.ident = false;
            o.liquid = true;
            spec_corot(o, mu, lam, J, Jk);
            break;
        case MPM_MAT_ELASTOPLASTIC:
        case MPM_MAT_SNOW:
            if (m.kind == MPM_MAT_ELASTOPLASTIC && (m.flags & MPM_MATF_VON_MISES)) {
                // elasto_plastic.py:70-84
                float Sc[3], de[3], e[3];
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    Sc[k] = fmaxf(s[k], 0.05f);
                    de[k] = s[k] > 0.05f ? 1.f / s[k] : 0.f;
                    e[k] = logf(Sc[k]);
                }
                const float mean = (e[0] + e[1] + e[2]) * (1.f / 3.f);
                const float eh[3] = {e[0] - mean, e[1] - mean, e[2] - mean};
                const float nn = sqrtf(eh[0] * eh[0] + eh[1] * eh[1] + eh[2] * eh[2] + eps);
                const float tau = m.vm_threshold * (m.mu / mu);
                if (nn - tau > 0.f) {
                    const float r = tau / nn;
#pragma unroll
                    for (int i = 0; i < 3; ++i) o.g[i] = expf(mean + r * eh[i]);
#pragma unroll
                    for (int i = 0; i < 3; ++i) {
#pragma unroll
                        for (int k = 0; k < 3; ++k) {
                            const float dedk = (1.f / 3.f) + r * ((i == k ? 1.f : 0.f) - (1.f / 3.f)) -
                                               (r / (nn * nn)) * eh[i] * eh[k];
                            o.Dg[i][k] = o.g[i] * dedk * de[k];
                            o.DDg[i][k] = ddiff_log(s[i], s[k], Sc[i], Sc[k], r, o.g[k]);
                        }
                        o.dg_dmu[i] = -o.g[i] * eh[i] * tau / (nn * mu);
                    }
                } else {
                    spec_ident(o, s);
                }
                spec_corot(o, mu, lam, J, Jk);
            } else {
                // clamp (elasto_plastic.py:86-90, snow.py:62-70)
                bool fr[3];
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    o.g[i] = fminf(fmaxf(s[i], m.clamp_lo), m.clamp_hi);
                    fr[i] = s[i] > m.clamp_lo && s[i] < m.clamp_hi;
                }
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        o.Dg[i][k] = (i == k && fr[i]) ? 1.f : 0.f;
                        const float den = s[i] - s[k];
                        o.DDg[i][k] = den != 0.f ? (o.g[i] - o.g[k]) / den : (fr[i] ? 1.f : 0.f);
                    }
                if (m.kind == MPM_MAT_SNOW) {
                    // Jp_new = Jp prod s / g; stress hardened by h = exp(10 (1 - Jp)) (snow.py:75-79)
                    const float h = expf(10.f * (1.f - Jp));
                    const float ratio = (s[0] / o.g[0]) * (s[1] / o.g[1]) * (s[2] / o.g[2]);
                    const float Jpn = Jp * ratio;
#pragma unroll
                    for (int i = 0; i < 3; ++i) o.dJpn_ds[i] = fr[i] ? 0.f : Jpn / s[i];
                    o.dJpn_dJp = ratio;
                    spec_corot(o, mu * h, lam * h, J, Jk);
#pragma unroll
                    for (int i = 0; i < 3; ++i) {
                        o.dp_dJp[i] = -10.f * o.p[i];
                        o.dp_dmu[i] *= h;
                        o.dp_dlam[i] *= h;
                    }
                } else {
                    spec_corot(o, mu, lam, J, Jk);
                }
            }
            break;
        case MPM_MAT_SAND:
        default: {
            // sand.py:51-89: ls = log S_new; p_i = 2 mu ls_i + lam sum(ls) (the stress
            // U diag(center) V^T F_new^T is U diag(center * S_new) U^T)
            float Sc[3], de[3], e[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                Sc[k] = fmaxf(fabsf(s[k]), 1e-4f);
                de[k] = fabsf(s[k]) > 1e-4f ? 1.f / s[k] : 0.f;
                e[k] = logf(Sc[k]);
            }
            const float tr = e[0] + e[1] + e[2] + Jp;
            const float eh[3] = {e[0] - tr / 3.f, e[1] - tr / 3.f, e[2] - tr / 3.f};
            const float nn = sqrtf(eh[0] * eh[0] + eh[1] * eh[1] + eh[2] * eh[2] + eps);
            const float q = (3.f * lam + 2.f * mu) / (2.f * mu) * m.sand_alpha;
            const float dq_dmu = m.sand_alpha * (-3.f * lam / (2.f * mu * mu));
            const float dq_dlam = m.sand_alpha * 3.f / (2.f * mu);
            if (tr >= 0.f) {  // expansion: S_new = I, Jp_new = tr
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    o.g[i] = 1.f;
                    o.p[i] = 0.f;
                    o.dp_dmu[i] = o.dp_dlam[i] = 0.f;
                    o.dJpn_ds[i] = de[i];
#pragma unroll
                    for (int k = 0; k < 3; ++k) o.Dp[i][k] = o.DDp[i][k] = 0.f;
                }
                o.dJpn_dJp = 1.f;
                break;
            }
            o.dJpn_dJp = 0.f;  // Jp_new = 0
            const bool y = nn + q * tr > 0.f;
            const float kap = y ? -q * tr / nn : 1.f;
            float ls[3], dls[3][3], dls_dJp[3], dls_dq[3];
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                ls[i] = y ? tr / 3.f + kap * eh[i] : e[i];
#pragma unroll
                for (int k = 0; k < 3; ++k)
                    dls[i][k] = y ? (1.f / 3.f) - q * (eh[i] / nn + (tr / nn) * ((i == k ? 1.f : 0.f) - (1.f / 3.f)) -
                                                       (tr / (nn * nn * nn)) * eh[i] * (eh[k] + Jp / 3.f))
                                  : (i == k ? 1.f : 0.f);
                dls_dJp[i] = y ? (1.f / 3.f) - q * (eh[i] / nn - tr / (3.f * nn) - tr * Jp / (3.f * nn * nn * nn) * eh[i])
                               : 0.f;
                dls_dq[i] = y ? -(tr / nn) * eh[i] : 0.f;
            }
            const float lsum = ls[0] + ls[1] + ls[2];
            const float dqs = dls_dq[0] + dls_dq[1] + dls_dq[2];
            const float djs = dls_dJp[0] + dls_dJp[1] + dls_dJp[2];
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                o.g[i] = expf(ls[i]);
                o.p[i] = 2.f * mu * ls[i] + lam * lsum;
                o.dg_dJp[i] = o.g[i] * dls_dJp[i];
                o.dg_dmu[i] = o.g[i] * dls_dq[i] * dq_dmu;
                o.dg_dlam[i] = o.g[i] * dls_dq[i] * dq_dlam;
                o.dp_dJp[i] = 2.f * mu * dls_dJp[i] + lam * djs;
                const float dpq = 2.f * mu * dls_dq[i] + lam * dqs;
                o.dp_dmu[i] = 2.f * ls[i] + dpq * dq_dmu;
                o.dp_dlam[i] = lsum + dpq * dq_dlam;
            }
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const float colsum = (dls[0][k] + dls[1][k] + dls[2][k]) * de[k];
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    o.Dg[i][k] = o.g[i] * dls[i][k] * de[k];
                    o.Dp[i][k] = 2.f * mu * dls[i][k] * de[k] + lam * colsum;
                    o.DDg[i][k] = ddiff_log(s[i], s[k], Sc[i], Sc[k], kap, o.g[k]);
                    const float den = s[i] - s[k];
                    o.DDp[i][k] = den != 0.f ? 2.f * mu * kap * log1pf((Sc[i] - Sc[k]) / Sc[k]) / den
                                             : 2.f * mu * kap / s[k];
                }
            }
            break;
        }
    }
}

// Adds the adjoint of F_tmp for the adjoints Gb of F_new, Jpnb of Jp_new and Pb of the
// material's stress; sets Jpb (adjoint of the previous Jp) and adds to mub, lamb.
__device__ void material_adjoint(const mpm_material& m, float mu, float lam, float eps, const float* U, const float* s,
                                 const float* V, float Jp, const float* Gb, float Jpnb, const float* Pb, float* Ftb,
                                 float& Jpb, float& mub, float& lamb) {
    Spec o;
    material_spectral(m, mu, lam, eps, s, Jp, o);
    float X[3][3], Z[3][3], T[3][3];
    // X = U^T Gb V
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            T[i][j] = Gb[i * 3 + 0] * V[0 * 3 + j] + Gb[i * 3 + 1] * V[1 * 3 + j] + Gb[i * 3 + 2] * V[2 * 3 + j];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) X[i][j] = U[0 * 3 + i] * T[0][j] + U[1 * 3 + i] * T[1][j] + U[2 * 3 + i] * T[2][j];
    // Z = U^T sym(Pb) U
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            float acc = 0.f;
#pragma unroll
            for (int k = 0; k < 3; ++k) acc += 0.5f * (Pb[i * 3 + k] + Pb[k * 3 + i]) * U[k * 3 + j];
            T[i][j] = acc;
        }
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) Z[i][j] = U[0 * 3 + i] * T[0][j] + U[1 * 3 + i] * T[1][j] + U[2 * 3 + i] * T[2][j];
    const bool use_x = !(o.ident || o.liquid);
    float sbar[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float acc = Jpnb * o.dJpn_ds[k];
#pragma unroll
        for (int i = 0; i < 3; ++i) acc += Z[i][i] * o.Dp[i][k] + (use_x ? X[i][i] * o.Dg[i][k] : 0.f);
        sbar[k] = acc;
    }
    Jpb = Jpnb * o.dJpn_dJp;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        Jpb += Z[i][i] * o.dp_dJp[i] + (use_x ? X[i][i] * o.dg_dJp[i] : 0.f);
        mub += Z[i][i] * o.dp_dmu[i] + (use_x ? X[i][i] * o.dg_dmu[i] : 0.f);
        lamb += Z[i][i] * o.dp_dlam[i] + (use_x ? X[i][i] * o.dg_dlam[i] : 0.f);
    }
    if (o.liquid) {
        // F_new = c I, c = J^(1/3): J_bar = tr(Gb) c / (3 J)
        const float J = s[0] * (s[1] * s[2]);
        const float Jb = (Gb[0] + Gb[4] + Gb[8]) * cbrtf(J) / (3.f * J);
        sbar[0] += Jb * s[1] * s[2];
        sbar[1] += Jb * s[0] * s[2];
        sbar[2] += Jb * s[0] * s[1];
    }
    float Y[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            if (i == j) {
                Y[i][j] = sbar[i];
                continue;
            }
            const float ss = s[i] + s[j];
            const bool ok = fabsf(ss) > 1e-12f;
            const float G = ok ? (o.g[i] + o.g[j]) / ss : 0.f;
            const float Gam = ok ? o.DDp[i][j] / ss : 0.f;
            float y = 2.f * Z[i][j] * s[j] * Gam;
            if (use_x) y += 0.5f * ((X[i][j] + X[j][i]) * o.DDg[i][j] + (X[i][j] - X[j][i]) * G);
            Y[i][j] = y;
        }
    // F_tmp_bar += U Y V^T (+ Gb where F_new = F_tmp)
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) T[i][j] = Y[i][0] * V[j * 3 + 0] + Y[i][1] * V[j * 3 + 1] + Y[i][2] * V[j * 3 + 2];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            Ftb[i * 3 + j] += U[i * 3 + 0] * T[0][j] + U[i * 3 + 1] * T[1][j] + U[i * 3 + 2] * T[2][j] +
                              (o.ident ? Gb[i * 3 + j] : 0.f);
}

// ---- adjoint of p2g, the materials and compute_F_tmp (mpm_solver.py:261-389)
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
    const float mu = par.mu_p ? ((m.kind == MPM_MAT_LIQUID && m.mu == 0.f) ? 0.f : par.mu_p[s]) : m.mu;
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
    float U[9], Sg[3], V[9];
    svd3(Ft, U, Sg, V);
    const float J = Sg[0] * (Sg[1] * Sg[2]);
    const float Jp = S[MPM_CH_JP * st + s];
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
    // the forward's stress (the same return mapping and stress code as p2g)
    float P[9], Fn[9], Jpn;
    constitutive(m, mu, lam, I.eps, J, Ft, U, Sg, V, Jp, Fn, Jpn, P);
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
    // the return mapping, the stress and the SVD (adjoints of F_new and Jp_new come in with adj)
    float* xo = adj + (int64_t)MPM_CH_X * st;
    float* vo = adj + (int64_t)MPM_CH_V * st;
    float* co = adj + (int64_t)MPM_CH_C * st;
    float* fo = adj + (int64_t)MPM_CH_F * st;
    float* jo = adj + (int64_t)MPM_CH_JP * st;
    float Gb[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) Gb[k] = fo[k * st + s];
    float Jpb = 0.f;
    material_adjoint(m, mu, lam, I.eps, U, Sg, V, Jp, Gb, jo[s], Pb, Ftb, Jpb, mub, lamb);
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
    jo[s] = Jpb;
    // inviscid Liquid never reads its mu (liquid.py:47-48): no gradient flows to it
    lame_bar[s] += (m.kind == MPM_MAT_LIQUID && m.mu == 0.f) ? 0.f : mub;
    lame_bar[st + s] += lamb;
}
