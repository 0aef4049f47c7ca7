// CPML and coefficient helpers shared by the fused-step kernels
// (stencil_fused.cu, stencil_tile.cu).  Reference: cpml.py:343-516 for the
// psi recursion and its correction.
#pragma once
#include "fitb_common.cuh"

#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace fitb {

namespace {

template <typename T>
struct FCoef {
    T ax, ay, az, bx, by, bz;
};

template <typename T>
__device__ __forceinline__ void load_coef3(FCoef<T>& c, const T* __restrict__ a, const T* __restrict__ b, long long o,
                                           long long vol) {
    c.ax = __ldg(a + o);
    c.ay = __ldg(a + vol + o);
    c.az = __ldg(a + 2 * vol + o);
    c.bx = __ldg(b + o);
    c.by = __ldg(b + vol + o);
    c.bz = __ldg(b + 2 * vol + o);
}

// H coefficients of one cell in the handle's storage: the field dtype, or
// the compact 16-bit copies times their per-component scales (decoded as
// the stream kernels decode them).
template <typename T>
__device__ __forceinline__ void load_coefH_stored(FCoef<T>& c, const StencilArgs<T>& p, long long o, long long vol) {
    if (p.coef_kind == kCoefNative) {
        load_coef3(c, p.aH, p.bH, o, vol);
        return;
    }
    const unsigned short *qa = p.cq[2], *qb = p.cq[3];
    auto dec = [&](unsigned short u) {
        return p.coef_kind == kCoefF16 ? __half2float(__ushort_as_half(u)) : __bfloat162float(__ushort_as_bfloat16(u));
    };
    c.ax = (T)dec(qa[o]) * (T)p.cs[8];
    c.ay = (T)dec(qa[vol + o]) * (T)p.cs[9];
    c.az = (T)dec(qa[2 * vol + o]) * (T)p.cs[10];
    c.bx = (T)dec(qb[o]) * (T)p.cs[12];
    c.by = (T)dec(qb[vol + o]) * (T)p.cs[13];
    c.bz = (T)dec(qb[2 * vol + o]) * (T)p.cs[14];
}

__device__ __forceinline__ long long slab_at(const FaceDev& f, int l, int i, int j, int k) {
    const int a = (f.axis == 0) ? l : i;
    const int b = (f.axis == 1) ? l : j;
    const int c = (f.axis == 2) ? l : k;
    return ((long long)a * f.dJ + b) * f.pk + c;
}

template <typename T>
__device__ __forceinline__ unsigned mask_jk(const StencilArgs<T>& p, int j, int k) {
    unsigned m = 0;
    for (int q = 0; q < p.nfaces; ++q) {
        const FaceDev& f = p.f[q];
        const int c = f.axis == 1 ? j : k;
        if (f.axis != 0 && (unsigned)(c - f.lo) < (unsigned)f.n) m |= 1u << q;
    }
    return m;
}

template <typename T>
__device__ __forceinline__ unsigned mask_i(const StencilArgs<T>& p, int i) {
    unsigned m = 0;
    for (int q = 0; q < p.nfaces; ++q) {
        const FaceDev& f = p.f[q];
        if (f.axis == 0 && (unsigned)(i - f.lo) < (unsigned)f.n) m |= 1u << q;
    }
    return m;
}

// CPML of the E update of one cell (cpml.py:343-430): psi_next = air *
// (b psi_old + c d), E -/+= beta (ck d + psi_next) on the two transverse
// components, faces in `mask` order.  d1/d2 per face axis as in the
// two-pass kernels.  `store`: write psi_next (owned cells only).
template <typename T>
__device__ __forceinline__ void cpml_E(const StencilArgs<T>& p, unsigned mask, int b, int i, int j, int k, T dx1,
                                       T dx2, T dy1, T dy2, T dz1, T dz2, const FCoef<T>& c, T& ex, T& ey, T& ez,
                                       bool store) {
    while (mask) {
        const int q = __ffs(mask) - 1;
        mask &= mask - 1;
        const FaceDev& f = p.f[q];
        const int coord = (f.axis == 0) ? i : ((f.axis == 1) ? j : k);
        const int l = coord - f.lo;
        const long long s = slab_at(f, l, i, j, k);
        const T* bcc = static_cast<const T*>(f.bcc);
        const T cb = bcc[l], cc = bcc[f.n + l], cck = bcc[2 * f.n + l];
        const long long off = (long long)b * 4 * f.slab;
        const T* psi = static_cast<const T*>(f.psi) + off;
        T* psin = static_cast<T*>(f.psi_next) + off;
        const T d1 = f.axis == 0 ? dx1 : (f.axis == 1 ? dy1 : dz1);
        const T d2 = f.axis == 0 ? dx2 : (f.axis == 1 ? dy2 : dz2);
        T p1 = psi[s] * cb;
        p1 = p1 + cc * d1;
        if (!f.air[s]) p1 = T(0);
        T p2 = psi[f.slab + s] * cb;
        p2 = p2 + cc * d2;
        if (!f.air[f.slab + s]) p2 = T(0);
        if (store) {
            psin[s] = p1;
            psin[f.slab + s] = p2;
        }
        if (f.axis == 0) {
            ey = ey + c.by * (cck * d1 + p1);
            ez = ez - c.bz * (cck * d2 + p2);
        } else if (f.axis == 1) {
            ex = ex - c.bx * (cck * d1 + p1);
            ez = ez + c.bz * (cck * d2 + p2);
        } else {
            ex = ex + c.bx * (cck * d1 + p1);
            ey = ey - c.by * (cck * d2 + p2);
        }
    }
}

// CPML of the H update of one cell (cpml.py:432-516); psi components 2, 3.
template <typename T>
__device__ __forceinline__ void cpml_H(const StencilArgs<T>& p, unsigned mask, int b, int i, int j, int k, T dx1,
                                       T dx2, T dy1, T dy2, T dz1, T dz2, const FCoef<T>& c, T& hx, T& hy, T& hz) {
    while (mask) {
        const int q = __ffs(mask) - 1;
        mask &= mask - 1;
        const FaceDev& f = p.f[q];
        const int coord = (f.axis == 0) ? i : ((f.axis == 1) ? j : k);
        const int l = coord - f.lo;
        const long long s = slab_at(f, l, i, j, k);
        const T* bcc = static_cast<const T*>(f.bcc);
        const T cb = bcc[l], cc = bcc[f.n + l], cck = bcc[2 * f.n + l];
        const long long off = (long long)b * 4 * f.slab;
        const T* psi = static_cast<const T*>(f.psi) + off;
        T* psin = static_cast<T*>(f.psi_next) + off;
        const T d1 = f.axis == 0 ? dx1 : (f.axis == 1 ? dy1 : dz1);
        const T d2 = f.axis == 0 ? dx2 : (f.axis == 1 ? dy2 : dz2);
        const long long s1 = 2 * f.slab + s, s2 = 3 * f.slab + s;
        T p1 = psi[s1] * cb;
        p1 = p1 + cc * d1;
        if (!f.air[s1]) p1 = T(0);
        psin[s1] = p1;
        T p2 = psi[s2] * cb;
        p2 = p2 + cc * d2;
        if (!f.air[s2]) p2 = T(0);
        psin[s2] = p2;
        if (f.axis == 0) {
            hy = hy - c.by * (cck * d1 + p1);
            hz = hz + c.bz * (cck * d2 + p2);
        } else if (f.axis == 1) {
            hx = hx + c.bx * (cck * d1 + p1);
            hz = hz - c.bz * (cck * d2 + p2);
        } else {
            hx = hx - c.bx * (cck * d1 + p1);
            hy = hy + c.by * (cck * d2 + p2);
        }
    }
}

}  // namespace

}  // namespace fitb
