// wd_adjoint.cuh -- derivatives of one contact, for the reverse pass of a step.
//
// The contact laws of wd_device.cuh (pair: src/compute_rhs_kernel.cu:150-204; walls:
// :114-146; damping: :41-47; the tangential spring extension) restated over a scalar
// type S that is either float or Dual<3> (a value plus three directional derivatives).
// Every operation on the value part is the float operation of the forward code in the
// same order (fmaf where the forward uses fmaf), so the values, and therefore every
// branch the forward took (clamp at max_force, Coulomb slip, the viscous cap, the
// 1e-8 cutoff), are the forward's own: the derivatives are those of the branch that
// ran (the frozen contact / stick-slip / clamp pattern of the step).
//
// Four passes over one contact seed three inputs each -- (d or x), (v_rel or v), the
// stored spring xi, and the parameters (mu, ln e, k_n) -- and give the Jacobian of the
// contact's force and of its new spring, column block by column block.
#pragma once

#include "wd_device.cuh"

namespace wd {

template <int N>
struct Dual {
    float v;
    float d[N];
};

template <int N>
__device__ __forceinline__ Dual<N> dconst(float v) {
    Dual<N> r;
    r.v = v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = 0.f;
    return r;
}

template <int N>
__device__ __forceinline__ Dual<N> dseed(float v, int k) {
    Dual<N> r = dconst<N>(v);
    if (k >= 0 && k < N) r.d[k] = 1.f;
    return r;
}

template <int N>
__device__ __forceinline__ Dual<N> operator+(Dual<N> a, Dual<N> b) {
    Dual<N> r;
    r.v = a.v + b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(Dual<N> a, Dual<N> b) {
    Dual<N> r;
    r.v = a.v - b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(Dual<N> a) {
    Dual<N> r;
    r.v = -a.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(Dual<N> a, Dual<N> b) {
    Dual<N> r;
    r.v = a.v * b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator/(Dual<N> a, Dual<N> b) {
    Dual<N> r;
    r.v = a.v / b.v;
    const float inv = 1.f / b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * inv;
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> fma_(Dual<N> a, Dual<N> b, Dual<N> c) {
    Dual<N> r;
    r.v = fmaf(a.v, b.v, c.v);
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i] + c.d[i];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> sqrt_(Dual<N> a) {
    Dual<N> r;
    r.v = sqrtf(a.v);
    const float h = r.v > 0.f ? 0.5f / r.v : 0.f;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * h;
    return r;
}
// min / max follow the branch the values take (ties: the first argument, as fminf
// and fmaxf return either and the forward's value is the same).
template <int N>
__device__ __forceinline__ Dual<N> fmin_(Dual<N> a, Dual<N> b) { return b.v < a.v ? b : a; }
template <int N>
__device__ __forceinline__ Dual<N> fmax_(Dual<N> a, Dual<N> b) { return b.v > a.v ? b : a; }

// float overloads, so the same templates also evaluate plain values
__device__ __forceinline__ float fma_(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ float sqrt_(float a) { return sqrtf(a); }
__device__ __forceinline__ float fmin_(float a, float b) { return fminf(a, b); }
__device__ __forceinline__ float fmax_(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ float val(float a) { return a; }
template <int N>
__device__ __forceinline__ float val(const Dual<N>& a) { return a.v; }

template <class S>
__device__ __forceinline__ S lift(float v) { return S(v); }
template <>
__device__ __forceinline__ Dual<3> lift<Dual<3>>(float v) { return dconst<3>(v); }

// Contact parameters as differentiable scalars: mu, L = ln e, k_n, and k_t (2/7 k_n
// when derived from it, else the fixed physics.tangential_stiffness).
template <class S>
struct Theta {
    S mu, L, k, kt;
};

// reference src/compute_rhs_kernel.cu:41-47, as damping() in wd_device.cuh.
template <class S>
__device__ __forceinline__ S damping_t(const DevParams& P, const Theta<S>& th, float m) {
    if (P.restitution <= 0.f) return lift<S>(2.f) * sqrt_(lift<S>(m) * th.k);
    if (P.restitution >= 1.f) return lift<S>(0.f);
    const float pi = 3.14159265358979323846f;
    const S den = sqrt_(fma_(th.L, th.L, lift<S>(pi * pi)));
    return ((lift<S>(-2.f) * sqrt_(lift<S>(m) * th.k)) * th.L) / den;
}

template <class S>
struct ContactOut {
    S f[3];    // the contact's force on this grain
    S xi[3];   // its new spring (history mode)
};

// Tangential spring: spring_friction() of wd_device.cuh.
template <class S>
__device__ __forceinline__ void spring_t(const DevParams& P, const Theta<S>& th, const S vt[3],
                                         const S nrm[3], S limit, const S xi_in[3],
                                         ContactOut<S>& o) {
    S xi[3] = {xi_in[0], xi_in[1], xi_in[2]};
    S xn = xi[0] * nrm[0];
    xn = fma_(xi[1], nrm[1], xn);
    xn = fma_(xi[2], nrm[2], xn);
#pragma unroll
    for (int a = 0; a < 3; ++a) xi[a] = fma_(-xn, nrm[a], xi[a]);
    const S dt = lift<S>(P.dt);
#pragma unroll
    for (int a = 0; a < 3; ++a) xi[a] = fma_(dt, vt[a], xi[a]);
    S ft[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) ft[a] = -th.kt * xi[a];
    S ft_sq = ft[0] * ft[0];
    ft_sq = fma_(ft[1], ft[1], ft_sq);
    ft_sq = fma_(ft[2], ft[2], ft_sq);
    if (val(ft_sq) > val(limit) * val(limit)) {
        const S s = limit / sqrt_(ft_sq);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            ft[a] = ft[a] * s;
            xi[a] = xi[a] * s;
        }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        o.f[a] = o.f[a] + ft[a];
        o.xi[a] = xi[a];
    }
}

// viscous_friction() of wd_device.cuh (reference src/compute_rhs_kernel.cu:66-78).
template <class S>
__device__ __forceinline__ void viscous_t(const S vt[3], S limit, S c, ContactOut<S>& o) {
    S vt_sq = vt[0] * vt[0];
    vt_sq = fma_(vt[1], vt[1], vt_sq);
    vt_sq = fma_(vt[2], vt[2], vt_sq);
    const S v = sqrt_(vt_sq);
    if (val(v) < 1e-8f) return;
    const S mag = fmin_(limit, c * v);
#pragma unroll
    for (int a = 0; a < 3; ++a) o.f[a] = o.f[a] - (mag * vt[a]) / v;
}

// One pair contact seen from grain i: pair_force() of wd_device.cuh, inputs
// d = x_i - x_j, vr = v_i - v_j and the stored spring of i's row.
template <class S, bool HIST>
__device__ __forceinline__ void pair_t(const DevParams& P, const Theta<S>& th, const S d[3],
                                       const S vr[3], const S xi_in[3], float ri, float rj,
                                       float mi, float mj, ContactOut<S>& o) {
#pragma unroll
    for (int a = 0; a < 3; ++a) o.f[a] = o.xi[a] = lift<S>(0.f);
    S ns = d[0] * d[0];
    ns = fma_(d[1], d[1], ns);
    ns = fma_(d[2], d[2], ns);
    const S norm = sqrt_(ns);
    const S nrm[3] = {d[0] / norm, d[1] / norm, d[2] / norm};
    const float rmax = fmaxf(ri, rj), rmin = fminf(ri, rj);
    const S dist = (norm - lift<S>(rmax)) - lift<S>(rmin);
    const S fp = fmax_(lift<S>(0.f), fmin_(lift<S>(P.max_force), -th.k * dist));
#pragma unroll
    for (int a = 0; a < 3; ++a) o.f[a] = fp * nrm[a];
    const float msum = mi + mj;
    const float mred = (msum > 0.f) ? (mi * mj) / msum : 0.f;
    const S c = damping_t(P, th, mred);
    S vn = vr[0] * nrm[0];
    vn = fma_(vr[1], nrm[1], vn);
    vn = fma_(vr[2], nrm[2], vn);
    const S cvn = c * vn;
#pragma unroll
    for (int a = 0; a < 3; ++a) o.f[a] = o.f[a] - cvn * nrm[a];
    S vt[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) vt[a] = fma_(-vn, nrm[a], vr[a]);
    const S limit = th.mu * fp;
    if (HIST) {
        spring_t(P, th, vt, nrm, limit, xi_in, o);
    } else {
        viscous_t(vt, limit, c, o);
    }
}

// One wall contact (axis a; upper = false: the lower wall): wall_forces() of
// wd_device.cuh for that wall alone. Inputs x, v of the grain and its stored spring.
template <class S, bool HIST>
__device__ __forceinline__ void wall_t(const DevParams& P, const Theta<S>& th, const S x[3],
                                       const S v[3], const S xi_in[3], float ri, float mi, int a,
                                       bool upper, ContactOut<S>& o) {
#pragma unroll
    for (int b = 0; b < 3; ++b) o.f[b] = o.xi[b] = lift<S>(0.f);
    const S dl = upper ? (lift<S>(P.wall_hi[a]) - x[a]) - lift<S>(ri)
                       : (x[a] - lift<S>(P.wall_lo[a])) - lift<S>(ri);
    const S fl = fmax_(lift<S>(0.f), fmin_(lift<S>(P.max_force), -th.k * dl));
    o.f[a] = upper ? -fl : fl;
    if (!(val(dl) < 0.f)) return;
    const S c = damping_t(P, th, mi);
    o.f[a] = o.f[a] - c * v[a];
    S vt[3], nrm[3];
#pragma unroll
    for (int b = 0; b < 3; ++b) {
        vt[b] = b == a ? lift<S>(0.f) : v[b];
        nrm[b] = lift<S>(b == a ? (upper ? -1.f : 1.f) : 0.f);
    }
    const S limit = th.mu * fl;
    if (HIST) {
        spring_t(P, th, vt, nrm, limit, xi_in, o);
    } else {
        viscous_t(vt, limit, c, o);
    }
}

}  // namespace wd
