// Adjoint (reverse mode) of one rigid-body step, for differentiable
// rollouts.  The reference has no adjoint; this differentiates the B200 step
// as the following model, with the step's discrete structure frozen from its
// forward run:
//
//  * state per dynamic body: mass-frame centre c and orientation Q, linear
//    and angular velocity; parameters: inverse mass, inverse principal
//    inertia, shape friction coefficients;
//  * broadphase pairs, manifold membership and contact counts, friction
//    anchor choice, partition levels and every clamp / branch decision of
//    prep and PGS are piecewise constant (taken from the forward run; the PGS
//    branches are read back from the impulse tape);
//  * contact geometry moves rigidly with the bodies, as the persistent PCM
//    manifold keeps it: point j of a manager (shape0 body A, shape1 body B)
//    is the material point Pb = c_B + R_B lb_j of B (fixed in the world when
//    B is static), its normal n = R_B nb, and its separation
//    s_j + n0 . ((c_A + R_A la_j) - (c_B + R_B lb_j)) with la, lb, nb the
//    forward point and normal in the bodies' frames; friction anchors are
//    body-local (as the step keeps them);
//  * everything else is the step's own arithmetic: pre-integration (gravity,
//    damping), the world sqrt-inverse-inertia tensor C = R diag(sqrt I^-1) R^T,
//    contact / friction / distance rows (scene.cpp:7490-8510), the 4 + 1 PGS
//    passes (scene.cpp:8853-9148) and integration (scene.cpp:114-143,
//    10508-10707).
//
// One step's reverse pass (enqueue_adjoint_step) runs after the step was
// re-run forward with its impulse tape: integration, then the PGS passes in
// reverse (islands in parallel, partitions and passes in reverse, each
// manager's rows in reverse; deltas are rebuilt by undoing each update),
// then contact / friction / joint preparation, then the per-body tensor,
// pre-integration and parameter accumulation.
#include "solver_common.cuh"
#include <cfloat>

namespace fyzz::b200 {
namespace {

__device__ __forceinline__ void atomic_add3(float4* p, v3 v) {
    atomicAdd(&p->x, v.x); atomicAdd(&p->y, v.y); atomicAdd(&p->z, v.z);
}
__device__ __forceinline__ void atomic_addq(float4* p, qt q) {
    atomicAdd(&p->x, q.x); atomicAdd(&p->y, q.y); atomicAdd(&p->z, q.z); atomicAdd(&p->w, q.w);
}
__device__ __forceinline__ float4 f4(v3 v, float w = 0.0f) { return make_float4(v.x, v.y, v.z, w); }

// Adjoint of out = rot_sc(q, v) (v + w t + u x t, t = 2 u x v): accumulates
// into qb and returns the adjoint of v.
__device__ __forceinline__ v3 rot_sc_adj(qt q, v3 v, v3 g, qt& qb) {
    const v3 u = {q.x, q.y, q.z};
    const v3 t = vmul(vcross(u, v), 2.0f);
    v3 ub = vcross(t, g);
    const v3 tb = vadd(vmul(g, q.w), vcross(g, u));
    qb.w += vdot(t, g);
    ub = vadd(ub, vmul(vcross(v, tb), 2.0f));
    qb.x += ub.x; qb.y += ub.y; qb.z += ub.z;
    return vadd(g, vmul(vcross(tb, u), 2.0f));
}
// C v with C the symmetric tensor stored as three float4 columns.
struct Tensor { v3 c0, c1, c2; };
__device__ __forceinline__ Tensor load_tensor(const DevState& s, int32_t b) {
    if (b < 0) return {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    const float4* si = s.sb_sqrt_i + 3 * size_t(b);
    return {ld3(si[0]), ld3(si[1]), ld3(si[2])};
}
__device__ __forceinline__ v3 tmul(const Tensor& C, v3 v) {
    return {C.c0.x * v.x + C.c1.x * v.y + C.c2.x * v.z,
            C.c0.y * v.x + C.c1.y * v.y + C.c2.y * v.z,
            C.c0.z * v.x + C.c1.z * v.y + C.c2.z * v.z};
}
// Accumulate the adjoint of out = C v: Cb_ij += g_i v_j (rows of Cb).
__device__ __forceinline__ void tensor_adj_atomic(float4* Cb, v3 g, v3 v) {
    atomic_add3(Cb + 0, vmul(v, g.x));
    atomic_add3(Cb + 1, vmul(v, g.y));
    atomic_add3(Cb + 2, vmul(v, g.z));
}

// ---------------------------------------------------------------- integration
// Adjoint of integrate_q(pose, w, dt) (scene.cpp:114-143) for |w| below the
// clamp; returns the pose adjoint and accumulates the w adjoint.
__device__ qt integrate_q_adj(qt pose, v3 w, float dt, qt ob, v3& wb) {
    const float m2 = w.x * w.x + w.y * w.y + w.z * w.z;
    if (m2 == 0.0f) return ob;
    const float m = sqrtf(m2);
    const float v = dt * m * 0.5f;
    const float sv_ = sinf(v), cv = cosf(v);
    const float sn = sv_ / m, cs = cv;
    const qt a = {w.x * sn, w.y * sn, w.z * sn, 0.0f};
    const qt dq = qmul(a, pose);
    const qt nx = {dq.x + pose.x * cs, dq.y + pose.y * cs, dq.z + pose.z * cs, dq.w + pose.w * cs};
    const float len = sqrtf(nx.x * nx.x + nx.y * nx.y + nx.z * nx.z + nx.w * nx.w);
    const qt o = {nx.x / len, nx.y / len, nx.z / len, nx.w / len};
    const float od = o.x * ob.x + o.y * ob.y + o.z * ob.z + o.w * ob.w;
    const qt g = {(ob.x - o.x * od) / len, (ob.y - o.y * od) / len, (ob.z - o.z * od) / len,
                  (ob.w - o.w * od) / len};
    // nx = dq + pose * cs
    qt pb = {g.x * cs, g.y * cs, g.z * cs, g.w * cs};
    const float csb = g.x * pose.x + g.y * pose.y + g.z * pose.z + g.w * pose.w;
    // dq = a (x) pose
    const qt b = pose;
    const v3 ab = {b.w * g.x - b.z * g.y + b.y * g.z - b.x * g.w,
                   b.z * g.x + b.w * g.y - b.x * g.z - b.y * g.w,
                   -b.y * g.x + b.x * g.y + b.w * g.z - b.z * g.w};
    pb.x += a.w * g.x + a.z * g.y - a.y * g.z - a.x * g.w;
    pb.y += -a.z * g.x + a.w * g.y + a.x * g.z - a.y * g.w;
    pb.z += a.y * g.x - a.x * g.y + a.w * g.z - a.z * g.w;
    pb.w += a.x * g.x + a.y * g.y + a.z * g.z + a.w * g.w;
    // a = w * sn
    wb = vadd(wb, vmul(ab, sn));
    const float snb = w.x * ab.x + w.y * ab.y + w.z * ab.z;
    // sn = sin(v) / m, cs = cos(v), v = dt m / 2
    const float vb = snb * cv / m - csb * sv_;
    const float mb = -snb * sv_ / (m * m) + vb * dt * 0.5f;
    wb = vadd(wb, vmul(w, mb / m));
    return pb;
}

__global__ void k_adj_save_start(DevState s, AdjState A) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= s.n_bodies) return;
    A.x_c[b] = f4(mass_position(s, b));
    A.x_q[b] = stq(mass_orientation(s, b));
}

// Per-step scratch: body adjoints of the deltas, velocities and tensors.
__global__ void k_adj_clear_bodies(DevState s, AdjState A) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= s.n_bodies) return;
    const float4 z = make_float4(0, 0, 0, 0);
    A.dvm[b] = z; A.dwm[b] = z; A.dv[b] = z; A.dw[b] = z; A.v1[b] = z; A.w1[b] = z;
    A.C[3 * size_t(b)] = z; A.C[3 * size_t(b) + 1] = z; A.C[3 * size_t(b) + 2] = z;
    A.im[b] = 0.0f; A.iI[b] = z;
    A.rdv[b] = s.sb_dv[b]; A.rdw[b] = s.sb_dw[b];
}
// Per-step scratch of the rows.
__global__ void k_adj_clear_rows(DevState s, AdjState A) {
    const uint32_t nm = s.counters[kCntMan];
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < nm; m += stride) {
        float4* n4 = reinterpret_cast<float4*>(A.nrow + 4 * size_t(m));
        float4* f4p = reinterpret_cast<float4*>(A.frow + 4 * size_t(m));
        for (int k = 0; k < 16; ++k) { n4[k] = make_float4(0, 0, 0, 0); f4p[k] = make_float4(0, 0, 0, 0); }
        A.hd[m] = make_float4(0, 0, 0, 0);
        for (int k = 0; k < 4; ++k) { A.yn[4 * size_t(m) + k] = 0.0f; A.yf[4 * size_t(m) + k] = 0.0f; }
    }
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < s.n_joints; j += stride) {
        float4* j4 = reinterpret_cast<float4*>(A.jrow + j);
        for (int k = 0; k < 4; ++k) j4[k] = make_float4(0, 0, 0, 0);
        A.yj[j] = 0.0f;
    }
}

// Integration (k_integrate) in reverse: the end-of-step adjoints (c', Q',
// v', w') become adjoints of the start centre / orientation, of the
// pre-integrated velocities, of the position-pass and final deltas, and of C.
__global__ void k_adj_integrate(DevState s, AdjState A) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= s.n_bodies || !is_dyn(s, b)) return;
    const float dt = s.dt;
    const Tensor C = load_tensor(s, int32_t(b));
    const v3 w1 = ld3(s.sb_w[b]);
    const v3 mdw = ld3(s.sb_mdw[b]), fdw = ld3(s.sb_dw[b]);
    const v3 cb = ld3(A.c[b]);
    const qt Qb_out = ldq(A.q[b]);
    const v3 fvb = ld3(A.v[b]), fwb = ld3(A.w[b]);
    v3 v1b = vadd(vmul(cb, dt), fvb);          // c' = c + (v1 + dvm) dt ; v' = v1 + dv
    const v3 dvmb = vmul(cb, dt);
    const v3 dvb = fvb;
    v3 w1b = fwb;                              // w' = w1 + C dw
    const v3 dwb = tmul(C, fwb);
    float4* Cb = A.C + 3 * size_t(b);
    tensor_adj_atomic(Cb, fwb, fdw);
    const v3 mw = vadd(w1, tmul(C, mdw));      // Q' = integrate(Q, w1 + C dwm)
    v3 mwb = {0, 0, 0};
    const qt Qb = integrate_q_adj(ldq(A.x_q[b]), mw, dt, Qb_out, mwb);
    w1b = vadd(w1b, mwb);
    const v3 dwmb = tmul(C, mwb);
    tensor_adj_atomic(Cb, mwb, mdw);
    A.q[b] = stq(Qb);
    A.v1[b] = f4(v1b);
    A.w1[b] = f4(w1b);
    A.dvm[b] = f4(dvmb);
    A.dwm[b] = f4(dwmb);
    A.dv[b] = f4(dvb);
    A.dw[b] = f4(dwb);
}

// ---------------------------------------------------------------- PGS reverse
__device__ __forceinline__ int32_t joint_body(const DevState& s, uint32_t b) {
    return is_dyn(s, b) ? int32_t(b) : -1;
}
// Deltas (rebuilt backwards) and their adjoints, addressed by global body
// (RevGlobal) or by island-local slot in shared memory (RevLocal); handle -1
// is the static world.
struct RevGlobal {
    static constexpr bool kLocal = false;
    const AdjState& A;
    __device__ __forceinline__ void load(int32_t b, v3& v, v3& w, v3& vb, v3& wb) const {
        if (b < 0) { v = w = vb = wb = {0, 0, 0}; return; }
        v = ld3(A.rdv[b]); w = ld3(A.rdw[b]); vb = ld3(A.dv[b]); wb = ld3(A.dw[b]);
    }
    __device__ __forceinline__ void store(int32_t b, v3 v, v3 w, v3 vb, v3 wb) const {
        if (b < 0) return;
        A.rdv[b] = f4(v); A.rdw[b] = f4(w); A.dv[b] = f4(vb); A.dw[b] = f4(wb);
    }
};
struct RevLocal {
    static constexpr bool kLocal = true;
    float4* d;   // 4 per slot: delta v, delta w, their adjoints
    __device__ __forceinline__ void load(int32_t b, v3& v, v3& w, v3& vb, v3& wb) const {
        if (b < 0) { v = w = vb = wb = {0, 0, 0}; return; }
        v = ld3(d[4 * b]); w = ld3(d[4 * b + 1]); vb = ld3(d[4 * b + 2]); wb = ld3(d[4 * b + 3]);
    }
    __device__ __forceinline__ void store(int32_t b, v3 v, v3 w, v3 vb, v3 wb) const {
        if (b < 0) return;
        d[4 * b] = f4(v); d[4 * b + 1] = f4(w); d[4 * b + 2] = f4(vb); d[4 * b + 3] = f4(wb);
    }
};
__device__ __forceinline__ int32_t local_handle(uint32_t v) { return v == 0xffffu ? -1 : int32_t(v); }

// One row update in reverse.  Forward: y' = y + dl, av += n dl ima,
// bv -= n dl imb, aw += ra dl, bw -= rb dl, with dl from the row rule.
// Undoes the delta update (deltas before the row), accumulates the
// parameter adjoints of the update and returns the adjoint of dl.
struct RowAdj { v3 n, ra, rb; float ima, imb; };
__device__ __forceinline__ float undo_update(v3 n, v3 ra, v3 rb, float ima, float imb, float dl,
                                             v3& av, v3& aw, v3& bv, v3& bw,
                                             v3 avb, v3 awb, v3 bvb, v3 bwb, RowAdj& g) {
    const float da = dl * ima, db = dl * imb;
    av = {av.x - n.x * da, av.y - n.y * da, av.z - n.z * da};
    bv = {bv.x + n.x * db, bv.y + n.y * db, bv.z + n.z * db};
    aw = {aw.x - ra.x * dl, aw.y - ra.y * dl, aw.z - ra.z * dl};
    bw = {bw.x + rb.x * dl, bw.y + rb.y * dl, bw.z + rb.z * dl};
    const float nav = vdot(n, avb), nbv = vdot(n, bvb);
    g.n = vadd(g.n, vsub(vmul(avb, da), vmul(bvb, db)));
    g.ima += dl * nav;
    g.imb -= dl * nbv;
    g.ra = vadd(g.ra, vmul(awb, dl));
    g.rb = vsub(g.rb, vmul(bwb, dl));
    return ima * nav - imb * nbv + vdot(ra, awb) - vdot(rb, bwb);
}
// Adjoint of the relative velocity n.(av - bv) + aw.ra - bw.rb (deltas
// before the update) with adjoint vb_.
__device__ __forceinline__ void rel_adj(v3 n, v3 ra, v3 rb, v3 av, v3 aw, v3 bv, v3 bw, float gb,
                                        v3& avb, v3& awb, v3& bvb, v3& bwb, RowAdj& g) {
    avb = vadd(avb, vmul(n, gb));
    bvb = vsub(bvb, vmul(n, gb));
    awb = vadd(awb, vmul(ra, gb));
    bwb = vsub(bwb, vmul(rb, gb));
    g.n = vadd(g.n, vmul(vsub(av, bv), gb));
    g.ra = vadd(g.ra, vmul(aw, gb));
    g.rb = vsub(g.rb, vmul(bw, gb));
}

// Adds a row-gradient increment to its accumulator with 128-bit accesses
// (the row records are 16-byte aligned; fields the increment leaves at 0
// are unchanged).
template <class T> __device__ __forceinline__ void add_row(T& dst, const T& inc) {
    static_assert(sizeof(T) % 16 == 0 && alignof(T) == 16, "16-byte row record");
    float4* d = reinterpret_cast<float4*>(&dst);
    const float4* a = reinterpret_cast<const float4*>(&inc);
#pragma unroll
    for (int k = 0; k < int(sizeof(T) / 16); ++k) {
        float4 x = d[k];
        const float4 y = a[k];
        x.x += y.x; x.y += y.y; x.z += y.z; x.w += y.w;
        d[k] = x;
    }
}
template <class R>
__device__ void reverse_desc(const DevState& s, const AdjState& A, uint32_t d, uint32_t lid, int it, int pos,
                             const R& D) {
    const size_t cap = s.pair_cap;
    if (d < s.n_joints) {
        const JointRow r = s.jrow[d];
        int32_t b0, b1;
        if constexpr (R::kLocal) {
            b0 = local_handle(lid & 0xffffu); b1 = local_handle(lid >> 16);
        } else {
            b0 = joint_body(s, s.j_a[d]); b1 = joint_body(s, s.j_b[d]);
        }
        v3 av, aw, bv, bw, avb, awb, bvb, bwb;
        D.load(b0, av, aw, avb, awb);
        D.load(b1, bv, bw, bvb, bwb);
        const v3 ax = lv(r.axis), ja = lv(r.ang_a), jb = lv(r.ang_b);
        const float yn = s.tape_j[size_t(it) * s.n_joints + d];
        const float yo = it > 0 ? s.tape_j[size_t(it - 1) * s.n_joints + d] : 0.0f;
        const float dl = yn - yo;
        RowAdj g = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, 0.0f, 0.0f};
        const float dlb = undo_update(ax, ja, jb, r.ima, r.imb, dl, av, aw, bv, bw, avb, awb, bvb, bwb, g);
        const float ynb = A.yj[d] + dlb;               // y' = y + nd vm + cst
        const float nd = vdot(ax, vsub(av, bv)) + vdot(ja, aw) - vdot(jb, bw);
        const float ndb = r.vel_mult * ynb;
        rel_adj(ax, ja, jb, av, aw, bv, bw, ndb, avb, awb, bvb, bwb, g);
        JointRow o = {};
        o.axis[0] = g.n.x; o.axis[1] = g.n.y; o.axis[2] = g.n.z;
        o.ang_a[0] = g.ra.x; o.ang_a[1] = g.ra.y; o.ang_a[2] = g.ra.z;
        o.ang_b[0] = g.rb.x; o.ang_b[1] = g.rb.y; o.ang_b[2] = g.rb.z;
        o.ima = g.ima; o.imb = g.imb;
        o.vel_mult = nd * ynb;
        if (it < pos) o.constant = ynb; else o.unbiased = ynb;
        add_row(A.jrow[d], o);
        A.yj[d] = ynb - dlb;
        D.store(b0, av, aw, avb, awb);
        D.store(b1, bv, bw, bvb, bwb);
        return;
    }
    const uint32_t m = d - s.n_joints;
    const ManagerHeader hd = s.mh[m];
    const float ima = hd.ima, imb = hd.imb;
    int32_t h0, h1;
    if constexpr (R::kLocal) {
        h0 = local_handle(lid & 0xffffu); h1 = local_handle(lid >> 16);
    } else {
        h0 = hd.b0; h1 = hd.b1;
    }
    v3 av, aw, bv, bw, avb, awb, bvb, bwb;
    D.load(h0, av, aw, avb, awb);
    D.load(h1, bv, bw, bvb, bwb);
    // the manager's four tape slots of this pass and the previous one, and
    // its four running row adjoints, as 128-bit loads
    const float4 zero4 = make_float4(0, 0, 0, 0);
    const size_t slot = size_t(it) * cap + m;
    const float4* tn4 = reinterpret_cast<const float4*>(s.tape_n);
    const float4* tf4 = reinterpret_cast<const float4*>(s.tape_f);
    const float tn[4] = {tn4[slot].x, tn4[slot].y, tn4[slot].z, tn4[slot].w};
    float4 y4 = reinterpret_cast<float4*>(A.yn)[m];
    float yv[4] = {y4.x, y4.y, y4.z, y4.w};
    RowAdj hg = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, 0.0f, 0.0f};
    float nsumb = 0.0f, dfb = 0.0f;
    const bool friction = (it >= pos || pos - it <= 3) && hd.anchors;
    if (friction) {
        const bool prev_friction = it > 0 && (it - 1 >= pos || pos - (it - 1) <= 3);
        const float4 x4 = tf4[slot], xo4 = prev_friction ? tf4[slot - cap] : zero4;
        const float xt[4] = {x4.x, x4.y, x4.z, x4.w}, xto[4] = {xo4.x, xo4.y, xo4.z, xo4.w};
        float4 f4 = reinterpret_cast<float4*>(A.yf)[m];
        float fv[4] = {f4.x, f4.y, f4.z, f4.w};
        float nsum = 0.0f;
#pragma unroll
        for (uint32_t j = 0; j < 4; ++j)
            if (j < hd.count) nsum += tn[j];
        const float coeff = hd.anchors == 2 ? 0.5f : 1.0f;
        const float md = hd.df * coeff * nsum;
        float mdb = 0.0f;
#pragma unroll
        for (int k = 3; k >= 0; --k) {
            if (k >= int(2 * hd.anchors)) continue;
            const FrictionRow f = s.frow[4 * size_t(m) + k];
            const v3 t = lv(f.t), ra = lv(f.ra), rb = lv(f.rb);
            const float xn = xt[k];
            const float xo = xto[k];
            RowAdj g = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, 0.0f, 0.0f};
            const float dlb = undo_update(t, ra, rb, ima, imb, xn - xo, av, aw, bv, bw, avb, awb, bvb, bwb, g);
            const float xnb = fv[k] + dlb;
            float xob = -dlb;
            FrictionRow o = {};
            if (xn == md && md != 0.0f) {
                mdb += xnb;
            } else if (xn == -md && md != 0.0f) {
                mdb -= xnb;
            } else if (!(xn == 0.0f && md == 0.0f)) {
                // unclamped: x' = x + (target - bias - td) vm
                const float bias = it < pos ? f.bias : 0.0f;
                const float td = vdot(t, vsub(av, bv)) + vdot(aw, ra) - vdot(bw, rb);
                xob += xnb;
                o.target = f.vel_mult * xnb;
                if (it < pos) o.bias = -(f.vel_mult * xnb);
                o.vel_mult = (f.target - bias - td) * xnb;
                rel_adj(t, ra, rb, av, aw, bv, bw, -f.vel_mult * xnb, avb, awb, bvb, bwb, g);
            } else {
                mdb += xnb;   // clamped to a zero bound
            }
            o.t[0] = g.n.x; o.t[1] = g.n.y; o.t[2] = g.n.z;
            o.ra[0] = g.ra.x; o.ra[1] = g.ra.y; o.ra[2] = g.ra.z;
            o.rb[0] = g.rb.x; o.rb[1] = g.rb.y; o.rb[2] = g.rb.z;
            add_row(A.frow[4 * size_t(m) + k], o);
            hg.ima += g.ima; hg.imb += g.imb;
            fv[k] = xob;
        }
        reinterpret_cast<float4*>(A.yf)[m] = make_float4(fv[0], fv[1], fv[2], fv[3]);
        dfb += coeff * nsum * mdb;
        nsumb += hd.df * coeff * mdb;
    }
    const float4 yo4 = it > 0 ? tn4[slot - cap] : zero4;
    const float tno[4] = {yo4.x, yo4.y, yo4.z, yo4.w};
#pragma unroll
    for (int j = 3; j >= 0; --j) {
        if (j >= int(hd.count)) continue;
        const NormalRow r = s.nrow[4 * size_t(m) + j];
        const v3 n = lv(r.n), ra = lv(r.ra), rb = lv(r.rb);
        const float yn = tn[j];
        const float yo = tno[j];
        RowAdj g = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, 0.0f, 0.0f};
        const float dlb = undo_update(n, ra, rb, ima, imb, yn - yo, av, aw, bv, bw, avb, awb, bvb, bwb, g);
        const float ynb = yv[j] + dlb + nsumb;
        float yob = -dlb;
        NormalRow o = {};
        if (yn != 0.0f) {
            // y' = imp y + (-nvel vm + err)
            const float nvel = vdot(n, vsub(av, bv)) + vdot(aw, ra) - vdot(bw, rb);
            yob += r.imp_mult * ynb;
            o.imp_mult = yo * ynb;
            o.vel_mult = -nvel * ynb;
            if (it < pos) o.biased = ynb; else o.unbiased = ynb;
            rel_adj(n, ra, rb, av, aw, bv, bw, -r.vel_mult * ynb, avb, awb, bvb, bwb, g);
        }
        o.n[0] = g.n.x; o.n[1] = g.n.y; o.n[2] = g.n.z;
        o.ra[0] = g.ra.x; o.ra[1] = g.ra.y; o.ra[2] = g.ra.z;
        o.rb[0] = g.rb.x; o.rb[1] = g.rb.y; o.rb[2] = g.rb.z;
        add_row(A.nrow[4 * size_t(m) + j], o);
        hg.ima += g.ima; hg.imb += g.imb;
        yv[j] = yob;
    }
    reinterpret_cast<float4*>(A.yn)[m] = make_float4(yv[0], yv[1], yv[2], yv[3]);
    float4 h = A.hd[m];
    h.x += hg.ima; h.y += hg.imb; h.w += dfb;
    A.hd[m] = h;
    D.store(h0, av, aw, avb, awb);
    D.store(h1, bv, bw, bvb, bwb);
}

// Adds the position-pass delta adjoints of an island's bodies (once each).
__device__ __forceinline__ void inject_motion(const DevState& s, const AdjState& A, uint32_t d, uint32_t epoch) {
    int32_t b[2];
    if (d < s.n_joints) {
        b[0] = joint_body(s, s.j_a[d]); b[1] = joint_body(s, s.j_b[d]);
    } else {
        const ManagerHeader hd = s.mh[d - s.n_joints];
        b[0] = hd.b0; b[1] = hd.b1;
    }
    for (int k = 0; k < 2; ++k) {
        if (b[k] < 0) continue;
        if (atomicExch(&A.mark[b[k]], epoch) == epoch) continue;
        float4 v = A.dv[b[k]], w = A.dw[b[k]];
        const float4 mv = A.dvm[b[k]], mw = A.dwm[b[k]];
        v.x += mv.x; v.y += mv.y; v.z += mv.z;
        w.x += mw.x; w.y += mw.y; w.z += mw.z;
        A.dv[b[k]] = v; A.dw[b[k]] = w;
    }
}

// Reverse PGS sweep over island-local slots in shared memory: one warp per
// island of <= kSmallIsland descriptors (4 warps per block).
// One thread per tiny island (<= kRevTiny descriptors): its descriptors in
// reverse placed order (levels in reverse; a level's descriptors share no
// body), with the deltas and their adjoints in the thread's slice of shared
// memory.  Most islands of a loose pile are a box resting alone.
constexpr uint32_t kRevTiny = 8;
constexpr uint32_t kRevThreadBlock = 64;
__global__ void __launch_bounds__(kRevThreadBlock) k_adj_pgs_thread(DevState s, AdjState A) {
    __shared__ float4 sh[kRevThreadBlock][4 * (kRevTiny + 1)];
    const uint32_t ni = *s.n_isl;
    const int pos = s.pos_iters, vel = s.vel_iters < 1 ? 1 : s.vel_iters;
    float4* my = sh[threadIdx.x];
    const RevLocal D{my};
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t isl = blockIdx.x * blockDim.x + threadIdx.x; isl < ni; isl += stride) {
        const uint32_t begin = s.isl_begin[isl], end = s.isl_begin[isl + 1];
        if (end - begin > kRevTiny) continue;
        const uint32_t nb = s.isl_nbod[isl];
        const int32_t* ib = s.isl_bod + begin + isl;
        for (uint32_t l = 0; l < nb; ++l) {
            const int32_t g = ib[l];
            my[4 * l] = s.sb_dv[g]; my[4 * l + 1] = s.sb_dw[g];
            my[4 * l + 2] = A.dv[g]; my[4 * l + 3] = A.dw[g];
        }
        for (int it = pos + vel - 1; it >= 0; --it) {
            if (it == pos - 1)
                for (uint32_t l = 0; l < nb; ++l) {
                    const int32_t g = ib[l];
                    float4 v = my[4 * l + 2], w = my[4 * l + 3];
                    const float4 mv = A.dvm[g], mw = A.dwm[g];
                    v.x += mv.x; v.y += mv.y; v.z += mv.z;
                    w.x += mw.x; w.y += mw.y; w.z += mw.z;
                    my[4 * l + 2] = v; my[4 * l + 3] = w;
                }
            for (uint32_t i = end; i-- > begin;) reverse_desc(s, A, s.d_val2[i], s.d_lbod[i], it, pos, D);
        }
    }
}

constexpr uint32_t kRevWarps = 4;
__global__ void __launch_bounds__(kRevWarps * 32) k_adj_pgs_warp_smem(DevState s, AdjState A,
                                                                     const uint32_t* lvl_bound) {
    __shared__ float4 sh[kRevWarps][4 * (kSmallIsland + 1)];
    const uint32_t ni = *s.n_isl;
    const uint32_t lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const int pos = s.pos_iters, vel = s.vel_iters < 1 ? 1 : s.vel_iters;
    const RevLocal D{sh[wib]};
    for (uint32_t isl = warp; isl < ni; isl += nwarps) {
        const uint32_t begin = s.isl_begin[isl], end = s.isl_begin[isl + 1];
        if (end - begin > s.isl_warp || end - begin <= kRevTiny) continue;
        const uint32_t nlev = s.isl_end[isl];
        const uint32_t nb = s.isl_nbod[isl];
        const int32_t* ib = s.isl_bod + begin + isl;
        const uint32_t* bound = lvl_bound + begin + isl;
        for (uint32_t l = lane; l < nb; l += 32) {
            const int32_t g = ib[l];
            sh[wib][4 * l] = s.sb_dv[g]; sh[wib][4 * l + 1] = s.sb_dw[g];
            sh[wib][4 * l + 2] = A.dv[g]; sh[wib][4 * l + 3] = A.dw[g];
        }
        __syncwarp();
        for (int it = pos + vel - 1; it >= 0; --it) {
            if (it == pos - 1) {
                for (uint32_t l = lane; l < nb; l += 32) {
                    const int32_t g = ib[l];
                    float4 v = sh[wib][4 * l + 2], w = sh[wib][4 * l + 3];
                    const float4 mv = A.dvm[g], mw = A.dwm[g];
                    v.x += mv.x; v.y += mv.y; v.z += mv.z;
                    w.x += mw.x; w.y += mw.y; w.z += mw.z;
                    sh[wib][4 * l + 2] = v; sh[wib][4 * l + 3] = w;
                }
                __syncwarp();
            }
            for (int l = int(nlev) - 1; l >= 0; --l) {
                const uint32_t lb = bound[l], le = bound[l + 1];
                for (uint32_t i = lb + lane; i < le; i += 32) reverse_desc(s, A, s.d_val2[i], s.d_lbod[i], it, pos, D);
                __syncwarp();
            }
        }
        __syncwarp();
    }
}
// The same with one CTA per island of the forward's list 1: (isl_warp,
// isl_mid] descriptors.
__global__ void __launch_bounds__(128) k_adj_pgs_mid_smem(DevState s, AdjState A, const uint32_t* lvl_bound) {
    extern __shared__ float4 shm[];
    const uint32_t n_list = s.counters[list_counter(1)];
    const uint32_t* list = s.isl_list[1];
    const int pos = s.pos_iters, vel = s.vel_iters < 1 ? 1 : s.vel_iters;
    const RevLocal D{shm};
    for (uint32_t k = blockIdx.x; k < n_list; k += gridDim.x) {
        const uint32_t isl = list[k];
        const uint32_t begin = s.isl_begin[isl];
        const uint32_t nlev = s.isl_end[isl];
        const uint32_t nb = s.isl_nbod[isl];
        const int32_t* ib = s.isl_bod + begin + isl;
        const uint32_t* bound = lvl_bound + begin + isl;
        for (uint32_t l = threadIdx.x; l < nb; l += blockDim.x) {
            const int32_t g = ib[l];
            shm[4 * l] = s.sb_dv[g]; shm[4 * l + 1] = s.sb_dw[g];
            shm[4 * l + 2] = A.dv[g]; shm[4 * l + 3] = A.dw[g];
        }
        __syncthreads();
        for (int it = pos + vel - 1; it >= 0; --it) {
            if (it == pos - 1) {
                for (uint32_t l = threadIdx.x; l < nb; l += blockDim.x) {
                    const int32_t g = ib[l];
                    float4 v = shm[4 * l + 2], w = shm[4 * l + 3];
                    const float4 mv = A.dvm[g], mw = A.dwm[g];
                    v.x += mv.x; v.y += mv.y; v.z += mv.z;
                    w.x += mw.x; w.y += mw.y; w.z += mw.z;
                    shm[4 * l + 2] = v; shm[4 * l + 3] = w;
                }
                __syncthreads();
            }
            for (int l = int(nlev) - 1; l >= 0; --l) {
                const uint32_t lb = bound[l], le = bound[l + 1];
                for (uint32_t i = lb + threadIdx.x; i < le; i += blockDim.x)
                    reverse_desc(s, A, s.d_val2[i], s.d_lbod[i], it, pos, D);
                __syncthreads();
            }
        }
        __syncthreads();
    }
}

// Reverse PGS sweep on global memory: one CTA per island beyond isl_mid.
__global__ void __launch_bounds__(256) k_adj_pgs_block(DevState s, AdjState A, const uint32_t* lvl_bound) {
    const uint32_t ni = *s.n_isl;
    const uint32_t epoch = *A.epoch;
    const int pos = s.pos_iters, vel = s.vel_iters < 1 ? 1 : s.vel_iters;
    for (uint32_t isl = blockIdx.x; isl < ni; isl += gridDim.x) {
        const uint32_t begin = s.isl_begin[isl], end = s.isl_begin[isl + 1];
        if (end - begin <= s.isl_mid) continue;
        const uint32_t nlev = s.isl_end[isl];
        const uint32_t* bound = lvl_bound + begin + isl;
        for (int it = pos + vel - 1; it >= 0; --it) {
            if (it == pos - 1) {
                for (uint32_t i = begin + threadIdx.x; i < end; i += blockDim.x)
                    inject_motion(s, A, s.d_val2[i], epoch);
                __syncthreads();
            }
            for (int l = int(nlev) - 1; l >= 0; --l) {
                const uint32_t lb = bound[l], le = bound[l + 1];
                for (uint32_t i = lb + threadIdx.x; i < le; i += blockDim.x)
                    reverse_desc(s, A, s.d_val2[i], 0u, it, pos, RevGlobal{A});
                __syncthreads();
            }
        }
    }
}

// ---------------------------------------------------------------- prep reverse
struct BodyFrame { v3 c; qt q; v3 v, w; float im; Tensor C; bool dyn; };
__device__ __forceinline__ BodyFrame load_frame(const DevState& s, const AdjState& A, uint32_t body) {
    BodyFrame f;
    f.c = ld3(A.x_c[body]);
    f.q = ldq(A.x_q[body]);
    f.dyn = is_dyn(s, body);
    if (f.dyn) {
        f.v = ld3(s.sb_v[body]); f.w = ld3(s.sb_w[body]);
        f.im = s.b_inv[body].w;
        f.C = load_tensor(s, int32_t(body));
    } else {
        f.v = f.w = {0, 0, 0};
        f.im = 0.0f;
        f.C = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    }
    return f;
}
// Body-level adjoint accumulators of one manager side.
struct SideAdj { v3 c; qt q; v3 v, w; float im; v3 C0, C1, C2; };
__device__ __forceinline__ void tensor_adj(SideAdj& a, v3 g, v3 v) {
    a.C0 = vadd(a.C0, vmul(v, g.x));
    a.C1 = vadd(a.C1, vmul(v, g.y));
    a.C2 = vadd(a.C2, vmul(v, g.z));
}
__device__ __forceinline__ void flush_side(const AdjState& A, uint32_t body, const SideAdj& a) {
    atomic_add3(A.c + body, a.c);
    atomic_addq(A.q + body, a.q);
    atomic_add3(A.v1 + body, a.v);
    atomic_add3(A.w1 + body, a.w);
    atomicAdd(A.im + body, a.im);
    atomic_add3(A.C + 3 * size_t(body), a.C0);
    atomic_add3(A.C + 3 * size_t(body) + 1, a.C1);
    atomic_add3(A.C + 3 * size_t(body) + 2, a.C2);
}
// X(l) = c + R(q) l : accumulate the adjoint of a body-attached point.
__device__ __forceinline__ void point_adj(const BodyFrame& f, SideAdj& a, v3 l, v3 g) {
    a.c = vadd(a.c, g);
    (void)rot_sc_adj(f.q, l, g, a.q);
}

__global__ void k_adj_prep_contacts(DevState s, AdjState A) {
    const uint32_t nm = s.counters[kCntMan];
    const float inv_dt = 1.0f / s.dt;
    const float bias_coeff = 0.8f, bounce = -2.0f;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < nm; m += stride) {
        const uint32_t pair = s.man_list[m];
        uint32_t sh0, sh1;
        manager_bodies(s, pair, sh0, sh1);
        const uint32_t a0 = s.s_body[sh0], a1 = s.s_body[sh1];
        const BodyFrame FA = load_frame(s, A, a0), FB = load_frame(s, A, a1);
        const ManagerHeader hd = s.mh[m];
        const float4 m0 = s.s_mat[sh0], m1 = s.s_mat[sh1];
        const float rest_d = m0.w + m1.w;
        const float restitution = 0.5f * (m0.z + m1.z);
        SideAdj GA = {}, GB = {};
        const ContactPt* pts = s.pts + 4 * size_t(pair);
        const v3 n0 = lv(pts[0].n);
        v3 nb_ = {0, 0, 0};                        // adjoint of the manager normal
        const v3 nb_local = FB.dyn ? rotinv_sc(FB.q, n0) : n0;
        // ---- contact rows
        for (uint32_t j = 0; j < hd.count; ++j) {
            const NormalRow& gr = A.nrow[4 * size_t(m) + j];
            const v3 P = lv(pts[j].p);
            const v3 n = n0;
            const v3 rA = vsub(P, FA.c), rB = vsub(P, FB.c);
            const v3 raxn = vcross(rA, n), rbxn = vcross(rB, n);
            const v3 ra = tmul(FA.C, raxn), rb = tmul(FB.C, rbxn);
            const float vrel = vdot(n, vsub(FA.v, FB.v)) + (vdot(raxn, FA.w) - vdot(rbxn, FB.w));
            const float response = (FA.im + vdot(ra, ra)) + (FB.im + vdot(rb, rb));
            const float vm = response > 0.0f ? 1.0f / response : 0.0f;
            const float pen = pts[j].sep - rest_d;
            const float pen_dt = pen * inv_dt;
            const bool separated = pen >= 0.0f;
            const bool closing = -vrel > pen_dt;
            const bool bouncing = restitution > 0.0f && bounce > vrel && closing;
            const float pds = separated ? pen_dt : pen * (inv_dt * bias_coeff);
            const float sb = bouncing ? 0.0f : vm * pds;   // max(maxpen, pds) with maxpen = -1e32
            const float target = (bouncing ? -vrel * restitution : 0.0f) - vrel;
            // row outputs: n, ra, rb, vel_mult = vm, biased = target vm - sb,
            // unbiased = target vm - (bouncing ? 0 : max(sb, 0))
            const float bb = gr.biased, ub = gr.unbiased;
            const float targetb = vm * (bb + ub);
            float vmb = gr.vel_mult + target * (bb + ub);
            const float sbb = -bb - ((!bouncing && sb > 0.0f) ? ub : 0.0f);
            float penb = 0.0f;
            if (!bouncing) {
                vmb += pds * sbb;
                penb = vm * sbb * (separated ? inv_dt : inv_dt * bias_coeff);
            }
            const float vrelb = -(1.0f + (bouncing ? restitution : 0.0f)) * targetb;
            const float responseb = response > 0.0f ? -vm * vm * vmb : 0.0f;
            GA.im += responseb;
            GB.im += responseb;
            const v3 rab = vadd(lv(gr.ra), vmul(ra, 2.0f * responseb));
            const v3 rbb = vadd(lv(gr.rb), vmul(rb, 2.0f * responseb));
            nb_ = vadd(nb_, lv(gr.n));
            // vrel = n.(vA - vB) + raxn.wA - rbxn.wB
            nb_ = vadd(nb_, vmul(vsub(FA.v, FB.v), vrelb));
            GA.v = vadd(GA.v, vmul(n, vrelb));
            GB.v = vsub(GB.v, vmul(n, vrelb));
            v3 raxnb = vmul(FA.w, vrelb), rbxnb = vmul(FB.w, -vrelb);
            GA.w = vadd(GA.w, vmul(raxn, vrelb));
            GB.w = vsub(GB.w, vmul(rbxn, vrelb));
            // ra = C_A raxn, rb = C_B rbxn
            tensor_adj(GA, rab, raxn);
            tensor_adj(GB, rbb, rbxn);
            raxnb = vadd(raxnb, tmul(FA.C, rab));
            rbxnb = vadd(rbxnb, tmul(FB.C, rbb));
            // raxn = rA x n, rbxn = rB x n
            const v3 rAb = vcross(n, raxnb), rBb = vcross(n, rbxnb);
            nb_ = vadd(nb_, vadd(vcross(raxnb, rA), vcross(rbxnb, rB)));
            // rA = P - cA, rB = P - cB
            v3 Pb = vadd(rAb, rBb);
            GA.c = vsub(GA.c, rAb);
            GB.c = vsub(GB.c, rBb);
            // P (and the separation) through the rigid contact model
            const v3 sepb = vmul(n0, penb);        // s = s0 + n0.(Pa - Pb)
            const v3 la = rotinv_sc(FA.q, vsub(P, FA.c));
            if (FA.dyn) point_adj(FA, GA, la, sepb);
            if (FB.dyn) {
                const v3 lb = rotinv_sc(FB.q, vsub(P, FB.c));
                point_adj(FB, GB, lb, vsub(Pb, sepb));
            }
        }
        // ---- friction rows
        if (hd.anchors) {
            const FrictionHist h = s.cur.fric[pair];
            const v3 rel = vsub(FA.v, FB.v);
            const v3 n = n0;
            const float nr = vdot(rel, n);
            const v3 u = vsub(rel, {n.x * nr, n.y * nr, n.z * nr});
            const bool fallback = vlen2(u) <= 0.0001f;
            const v3 u0 = fallback ? (fabsf(n.x) < 0.70710678f ? v3{0.0f, -n.z, n.y} : v3{-n.y, n.x, 0.0f}) : u;
            const float ul = sqrtf(vlen2(u0));
            const v3 t0 = vmul(u0, 1.0f / ul);
            const v3 t1 = vcross(n, t0);
            v3 t0b = {0, 0, 0}, t1b = {0, 0, 0}, relb = {0, 0, 0};
            for (uint32_t k = 0; k < hd.anchors; ++k) {
                const v3 a0l = lv(h.a0[k]), a1l = lv(h.a1[k]);
                const v3 raK = rot_sc(FA.q, a0l), rbK = rot_sc(FB.q, a1l);
                // an anchor taken from this step's point P sits at P on both
                // bodies (lever arms P - c, zero error); a carried one is
                // body-local on each body
                const bool fresh = (h.meta >> (10 + k)) & 1u;
                const uint32_t src = (h.meta >> (12 + 2 * k)) & 3u;
                const v3 err = vsub(vadd(raK, FA.c), vadd(rbK, FB.c));
                v3 raKb = {0, 0, 0}, rbKb = {0, 0, 0}, errb = {0, 0, 0};
                for (int t = 0; t < 2; ++t) {
                    const FrictionRow& gf = A.frow[4 * size_t(m) + 2 * k + t];
                    const v3 tg = t == 0 ? t0 : t1;
                    const v3 ax0 = vcross(raK, tg), ax1 = vcross(rbK, tg);
                    const v3 j0 = tmul(FA.C, ax0), j1 = tmul(FB.C, ax1);
                    const float resp = (FA.im + vdot(j0, j0)) + (FB.im + vdot(j1, j1));
                    const float vmf = resp > 0.0f ? bias_coeff / resp : 0.0f;
                    v3 tgb = lv(gf.t);
                    // target = -(tg.rel + ax0.wA - ax1.wB)
                    const float tb = gf.target;
                    tgb = vsub(tgb, vmul(rel, tb));
                    relb = vsub(relb, vmul(tg, tb));
                    v3 ax0b = vmul(FA.w, -tb), ax1b = vmul(FB.w, tb);
                    GA.w = vsub(GA.w, vmul(ax0, tb));
                    GB.w = vadd(GB.w, vmul(ax1, tb));
                    // bias = tg.err / dt
                    tgb = vadd(tgb, vmul(err, gf.bias * inv_dt));
                    errb = vadd(errb, vmul(tg, gf.bias * inv_dt));
                    // vel_mult = 0.8 / resp
                    const float respb = resp > 0.0f ? -vmf / resp * gf.vel_mult : 0.0f;
                    GA.im += respb;
                    GB.im += respb;
                    const v3 j0b = vadd(lv(gf.ra), vmul(j0, 2.0f * respb));
                    const v3 j1b = vadd(lv(gf.rb), vmul(j1, 2.0f * respb));
                    tensor_adj(GA, j0b, ax0);
                    tensor_adj(GB, j1b, ax1);
                    ax0b = vadd(ax0b, tmul(FA.C, j0b));
                    ax1b = vadd(ax1b, tmul(FB.C, j1b));
                    // ax = r x tg
                    raKb = vadd(raKb, vcross(tg, ax0b));
                    rbKb = vadd(rbKb, vcross(tg, ax1b));
                    tgb = vadd(tgb, vadd(vcross(ax0b, raK), vcross(ax1b, rbK)));
                    if (t == 0) t0b = vadd(t0b, tgb); else t1b = vadd(t1b, tgb);
                }
                // err = (raK + cA) - (rbK + cB)
                raKb = vadd(raKb, errb);
                rbKb = vsub(rbKb, errb);
                GA.c = vadd(GA.c, errb);
                GB.c = vsub(GB.c, errb);
                if (fresh) {
                    // raK = P - cA, rbK = P - cB, P the (B-attached) contact point
                    const v3 Pb_ = vadd(raKb, rbKb);
                    GA.c = vsub(GA.c, raKb);
                    GB.c = vsub(GB.c, rbKb);
                    if (FB.dyn) {
                        const v3 P = lv(pts[src].p);
                        point_adj(FB, GB, rotinv_sc(FB.q, vsub(P, FB.c)), Pb_);
                    }
                } else {
                    if (FA.dyn) (void)rot_sc_adj(FA.q, a0l, raKb, GA.q);
                    if (FB.dyn) (void)rot_sc_adj(FB.q, a1l, rbKb, GB.q);
                }
            }
            // t1 = n x t0
            nb_ = vadd(nb_, vcross(t0, t1b));
            t0b = vadd(t0b, vcross(t1b, n));
            // t0 = u0 / |u0|
            const v3 u0b = vmul(vsub(t0b, vmul(t0, vdot(t0, t0b))), 1.0f / ul);
            if (!fallback) {
                // u = rel - n (n.rel)
                relb = vadd(relb, u0b);
                const float sb_ = -vdot(n, u0b);
                nb_ = vsub(nb_, vmul(u0b, nr));
                nb_ = vadd(nb_, vmul(rel, sb_));
                relb = vadd(relb, vmul(n, sb_));
            } else if (fabsf(n.x) < 0.70710678f) {
                nb_ = vadd(nb_, v3{0.0f, u0b.z, -u0b.y});
            } else {
                nb_ = vadd(nb_, v3{u0b.y, -u0b.x, 0.0f});
            }
            GA.v = vadd(GA.v, relb);
            GB.v = vsub(GB.v, relb);
        }
        // manager normal n = R_B nb (B dynamic)
        if (FB.dyn) (void)rot_sc_adj(FB.q, nb_local, nb_, GB.q);
        // header: ima, imb, sf, df
        const float4 h = A.hd[m];
        GA.im += h.x;
        GB.im += h.y;
        // sf = max(df, 0.5 (s0 + s1)), df = max(0, 0.5 (d0 + d1))
        float dfb = h.w, sfb = h.z;
        const float dsum = 0.5f * (m0.y + m1.y);
        const float dfr = smax(0.0f, dsum);
        const float ssum = 0.5f * (m0.x + m1.x);
        if (dfr < ssum) {
            atomicAdd(A.g_fs + sh0, 0.5f * sfb);
            atomicAdd(A.g_fs + sh1, 0.5f * sfb);
        } else {
            dfb += sfb;
        }
        if (0.0f < dsum) {
            atomicAdd(A.g_fd + sh0, 0.5f * dfb);
            atomicAdd(A.g_fd + sh1, 0.5f * dfb);
        }
        if (FA.dyn) flush_side(A, a0, GA);
        if (FB.dyn) flush_side(A, a1, GB);
    }
}

// Distance joints (k_prep_joints) in reverse.  Anchors are the body origins:
// origin = c - R(Q) u with u the mass-frame offset of the origin.
__global__ void k_adj_prep_joints(DevState s, AdjState A) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= s.n_joints) return;
    const uint32_t a = s.j_a[j], b = s.j_b[j];
    const BodyFrame F0 = load_frame(s, A, a), F1 = load_frame(s, A, b);
    const float inv_dt = 1.0f / s.dt;
    const v3 u0 = rotinv_sc(ldq(s.b_ml_q[a]), ld3(s.b_ml_p[a]));
    const v3 u1 = rotinv_sc(ldq(s.b_ml_q[b]), ld3(s.b_ml_p[b]));
    const v3 ra = vneg(rot_sc(F0.q, u0)), rb = vneg(rot_sc(F1.q, u1));
    const v3 off = vsub(vadd(F0.c, ra), vadd(F1.c, rb));
    const float dist = sqrtf(vdot(off, off));
    const bool degenerate = dist < 1.192092896e-07f;
    const v3 axis = degenerate ? v3{1, 0, 0} : vmul(off, 1.0f / dist);
    const v3 an0 = vcross(ra, axis), an1 = vcross(rb, axis);
    const v3 ja = F0.dyn ? tmul(F0.C, an0) : v3{0, 0, 0};
    const v3 jb = F1.dyn ? tmul(F1.C, an1) : v3{0, 0, 0};
    const float response = F0.im + F1.im + vdot(ja, ja) + vdot(jb, jb);
    const float rcp = 1.0f / response;
    const float speed = vdot(axis, vsub(F0.v, F1.v)) + vdot(an0, F0.w) - vdot(an1, F1.w);
    const float err = dist - s.j_len[j];
    const JointRow& g = A.jrow[j];
    SideAdj G0 = {}, G1 = {};
    // constant = -rcp (err/dt + speed), unbiased = -rcp speed, vel_mult = -rcp
    float rcpb = -g.vel_mult - g.constant * (err * inv_dt + speed) - g.unbiased * speed;
    const float errb = -rcp * g.constant * inv_dt;
    const float speedb = -rcp * (g.constant + g.unbiased);
    G0.im += g.ima;
    G1.im += g.imb;
    const float respb = -rcp * rcp * rcpb;
    G0.im += respb;
    G1.im += respb;
    v3 axisb = lv(g.axis);
    const v3 jab = vadd(lv(g.ang_a), vmul(ja, 2.0f * respb));
    const v3 jbb = vadd(lv(g.ang_b), vmul(jb, 2.0f * respb));
    v3 an0b = {0, 0, 0}, an1b = {0, 0, 0};
    if (F0.dyn) { tensor_adj(G0, jab, an0); an0b = tmul(F0.C, jab); }
    if (F1.dyn) { tensor_adj(G1, jbb, an1); an1b = tmul(F1.C, jbb); }
    // speed
    axisb = vadd(axisb, vmul(vsub(F0.v, F1.v), speedb));
    G0.v = vadd(G0.v, vmul(axis, speedb));
    G1.v = vsub(G1.v, vmul(axis, speedb));
    an0b = vadd(an0b, vmul(F0.w, speedb));
    an1b = vsub(an1b, vmul(F1.w, speedb));
    G0.w = vadd(G0.w, vmul(an0, speedb));
    G1.w = vsub(G1.w, vmul(an1, speedb));
    // an = r x axis
    v3 rab = vcross(axis, an0b), rbb = vcross(axis, an1b);
    axisb = vadd(axisb, vadd(vcross(an0b, ra), vcross(an1b, rb)));
    // axis = off / dist, err = dist - len
    v3 offb = {0, 0, 0};
    if (!degenerate) {
        offb = vmul(vsub(axisb, vmul(axis, vdot(axis, axisb))), 1.0f / dist);
        offb = vadd(offb, vmul(axis, errb));
    }
    G0.c = vadd(G0.c, offb);
    G1.c = vsub(G1.c, offb);
    rab = vadd(rab, offb);
    rbb = vsub(rbb, offb);
    // r = -R(Q) u
    if (F0.dyn) (void)rot_sc_adj(F0.q, u0, vneg(rab), G0.q);
    if (F1.dyn) (void)rot_sc_adj(F1.q, u1, vneg(rbb), G1.q);
    if (F0.dyn) flush_side(A, a, G0);
    if (F1.dyn) flush_side(A, b, G1);
}

// Per body: the tensor C = sum_k l_k r_k r_k^T (l = sqrt I^-1, r_k = R e_k)
// and pre-integration (v1 = lm (v + g dt), w1 = am w) in reverse; the
// start-of-step state adjoint and the parameter gradients.
__global__ void k_adj_bodies(DevState s, AdjState A) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= s.n_bodies || !is_dyn(s, b)) return;
    const float dt = s.dt;
    const qt Q = ldq(A.x_q[b]);
    const float4 inv = s.b_inv[b];
    const float l[3] = {sqrtf(inv.x), sqrtf(inv.y), sqrtf(inv.z)};
    const v3 Cb[3] = {ld3(A.C[3 * size_t(b)]), ld3(A.C[3 * size_t(b) + 1]), ld3(A.C[3 * size_t(b) + 2])};
    qt qb = ldq(A.q[b]);
    float4 iIb = A.iI[b];
    float lb_[3];
    for (int k = 0; k < 3; ++k) {
        const v3 e = {k == 0 ? 1.0f : 0.0f, k == 1 ? 1.0f : 0.0f, k == 2 ? 1.0f : 0.0f};
        const v3 r = rot_sc(Q, e);
        // l_k: r^T Cb r ; r_k: l_k (Cb + Cb^T) r
        const v3 Cr = {vdot(Cb[0], r), vdot(Cb[1], r), vdot(Cb[2], r)};
        const v3 CTr = vadd(vadd(vmul(Cb[0], r.x), vmul(Cb[1], r.y)), vmul(Cb[2], r.z));
        lb_[k] = vdot(r, Cr);
        const v3 rb = vmul(vadd(Cr, CTr), l[k]);
        (void)rot_sc_adj(Q, e, rb, qb);
    }
    iIb.x += l[0] > 0.0f ? lb_[0] / (2.0f * l[0]) : 0.0f;
    iIb.y += l[1] > 0.0f ? lb_[1] / (2.0f * l[1]) : 0.0f;
    iIb.z += l[2] > 0.0f ? lb_[2] / (2.0f * l[2]) : 0.0f;
    A.q[b] = stq(qb);
    const float4 d0 = s.b_dyn0[b];
    const float lm = smax(1.0f - d0.x * dt, 0.0f), am = smax(1.0f - d0.y * dt, 0.0f);
    A.v[b] = f4(vmul(ld3(A.v1[b]), lm));
    A.w[b] = f4(vmul(ld3(A.w1[b]), am));
    A.g_im[b] += A.im[b];
    float4 g = A.g_iI[b];
    g.x += iIb.x; g.y += iIb.y; g.z += iIb.z;
    A.g_iI[b] = g;
}

inline uint32_t grid_n(uint32_t n, uint32_t t, uint32_t cap) {
    const uint32_t g = (n + t - 1) / t;
    return g == 0 ? 1 : (g < cap ? g : cap);
}

__global__ void k_adj_next_epoch(AdjState A) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *A.epoch += 1u;
}

// Copies the live part of a contact-manager generation (its device count;
// the PCM caches only when dst has them).
__global__ void k_copy_set(ManagerSet dst, ManagerSet src, uint32_t cap) {
    const uint32_t n = min(*src.n, cap);
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        dst.key[i] = src.key[i];
        if (dst.cache) dst.cache[i] = src.cache[i];
        dst.fric[i] = src.fric[i];
        dst.count[i] = src.count[i];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *dst.n = *src.n;
}

}  // namespace

void enqueue_adjoint_save_start(const DevState& s, const AdjState& a, cudaStream_t st) {
    k_adj_save_start<<<grid_n(s.n_bodies, 256, 1u << 30), 256, 0, st>>>(s, a);
}

void enqueue_copy_set(const ManagerSet& dst, const ManagerSet& src, uint32_t cap, cudaStream_t st) {
    k_copy_set<<<grid_n(cap, 256, 148u * 8u), 256, 0, st>>>(dst, src, cap);
}

void enqueue_adjoint_step(const DevState& s, const AdjState& a, cudaStream_t st) {
    const uint32_t T = 256;
    k_adj_next_epoch<<<1, 32, 0, st>>>(a);
    k_adj_clear_bodies<<<grid_n(s.n_bodies, T, 1u << 30), T, 0, st>>>(s, a);
    k_adj_clear_rows<<<grid_n(s.pair_cap, T, 148u * 8u), T, 0, st>>>(s, a);
    k_adj_integrate<<<grid_n(s.n_bodies, T, 1u << 30), T, 0, st>>>(s, a);
    k_adj_pgs_thread<<<grid_n(s.desc_cap, kRevThreadBlock, 148u * 16u), kRevThreadBlock, 0, st>>>(s, a);
    k_adj_pgs_warp_smem<<<grid_n(s.desc_cap * 32u, kRevWarps * 32u, 148u * 8u), kRevWarps * 32u, 0, st>>>(
        s, a, s.lvl_bound);
    k_adj_pgs_mid_smem<<<grid_n(s.desc_cap, kSmallIsland + 1, 148u * 4u), 128,
                         4 * (kMidIsland + 1) * sizeof(float4), st>>>(s, a, s.lvl_bound);
    k_adj_pgs_block<<<grid_n(s.desc_cap, 1, 148u * 4u), 256, 0, st>>>(s, a, s.lvl_bound);
    k_adj_prep_contacts<<<grid_n(s.pair_cap, 128, 148u * 8u), 128, 0, st>>>(s, a);
    if (s.n_joints) k_adj_prep_joints<<<grid_n(s.n_joints, T, 1u << 30), T, 0, st>>>(s, a);
    k_adj_bodies<<<grid_n(s.n_bodies, T, 1u << 30), T, 0, st>>>(s, a);
}

}  // namespace fyzz::b200
