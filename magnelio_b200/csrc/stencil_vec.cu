// Vectorised leapfrog curl updates over flattened padded planes.
//
// Same arithmetic and in-thread order as stencil.cu and stencil_stream.cu
// (reference: numba_kernels.py:36-127, cpml.py:343-516); a different
// mapping of work to threads.  The rows j in [0, ny] of one padded plane
// are contiguous in memory (row stride nkp, a multiple of 4), so the plane
// is cut into vectors of VK consecutive entries and thread t of a warp owns
// vector 32 c + t of the plane: a warp reads 32 * VK * sizeof(T) contiguous
// bytes of every array with one 8- or 16-byte load per thread, and a vector
// never straddles two rows.  Each thread marches over a chunk of i planes
// with the next plane's loads in flight while it computes the current one,
// as the stream kernels do.
//
// Neighbours: along i from registers (the E update marches up, the H update
// down), along j by an aligned vector load one row away, along k by a warp
// shuffle of the neighbouring lane's first / last entry (the entry before
// vector q is the last entry of vector q-1 in memory, whichever row it is
// in, so the pad semantics of the layout are kept); only lane 0 (E) or lane
// 31 (H) loads that entry.  Entries with k > nz are pads: loaded, never
// stored.  The CPML faces a thread can meet are decided once per thread
// (y and z faces) and once per plane (x faces), so cells outside every slab
// run no face code.
#include "fitb_common.cuh"
#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace fitb {

namespace {

template <typename T, int VK>
struct Vt {
    T x[VK];
};

// Loads and stores of VK consecutive entries at an address aligned to
// VK * sizeof(T).
template <typename T, int VK>
__device__ __forceinline__ void ldg_v(Vt<T, VK>& r, const T* p) {
    if constexpr (sizeof(T) == 4 && VK == 4) {
        const float4 q = __ldg(reinterpret_cast<const float4*>(p));
        r.x[0] = q.x; r.x[1] = q.y; r.x[2] = q.z; r.x[3] = q.w;
    } else if constexpr (sizeof(T) == 4 && VK == 2) {
        const float2 q = __ldg(reinterpret_cast<const float2*>(p));
        r.x[0] = q.x; r.x[1] = q.y;
    } else {
        static_assert(sizeof(T) == 8 && VK == 2, "vector shape");
        const double2 q = __ldg(reinterpret_cast<const double2*>(p));
        r.x[0] = q.x; r.x[1] = q.y;
    }
}

template <typename T, int VK>
__device__ __forceinline__ void ld_v(Vt<T, VK>& r, const T* p) {
    if constexpr (sizeof(T) == 4 && VK == 4) {
        const float4 q = *reinterpret_cast<const float4*>(p);
        r.x[0] = q.x; r.x[1] = q.y; r.x[2] = q.z; r.x[3] = q.w;
    } else if constexpr (sizeof(T) == 4 && VK == 2) {
        const float2 q = *reinterpret_cast<const float2*>(p);
        r.x[0] = q.x; r.x[1] = q.y;
    } else {
        const double2 q = *reinterpret_cast<const double2*>(p);
        r.x[0] = q.x; r.x[1] = q.y;
    }
}

template <typename T, int VK>
__device__ __forceinline__ void st_v(T* p, const Vt<T, VK>& r) {
    if constexpr (sizeof(T) == 4 && VK == 4) {
        *reinterpret_cast<float4*>(p) = make_float4(r.x[0], r.x[1], r.x[2], r.x[3]);
    } else if constexpr (sizeof(T) == 4 && VK == 2) {
        *reinterpret_cast<float2*>(p) = make_float2(r.x[0], r.x[1]);
    } else {
        *reinterpret_cast<double2*>(p) = make_double2(r.x[0], r.x[1]);
    }
}

// Store the first n entries (n = VK: one vector store).
template <typename T, int VK>
__device__ __forceinline__ void st_v_n(T* p, const Vt<T, VK>& r, int n) {
    if (n >= VK) {
        st_v(p, r);
    } else {
#pragma unroll
        for (int e = 0; e < VK; ++e)
            if (e < n) p[e] = r.x[e];
    }
}

template <int CK>
__device__ __forceinline__ float unpack16(unsigned short u) {
    if constexpr (CK == kCoefF16)
        return __half2float(__ushort_as_half(u));
    else
        return __bfloat162float(__ushort_as_bfloat16(u));
}

template <typename T, int CK, int VK>
__device__ __forceinline__ void ldg_c(Vt<T, VK>& r, const T* __restrict__ native, const unsigned short* __restrict__ q16,
                                      float scale, long long o) {
    if constexpr (CK == kCoefNative) {
        ldg_v<T, VK>(r, native + o);
    } else if constexpr (VK == 4) {
        const ushort4 u = __ldg(reinterpret_cast<const ushort4*>(q16 + o));
        r.x[0] = (T)unpack16<CK>(u.x) * (T)scale;
        r.x[1] = (T)unpack16<CK>(u.y) * (T)scale;
        r.x[2] = (T)unpack16<CK>(u.z) * (T)scale;
        r.x[3] = (T)unpack16<CK>(u.w) * (T)scale;
    } else {
        const ushort2 u = __ldg(reinterpret_cast<const ushort2*>(q16 + o));
        r.x[0] = (T)unpack16<CK>(u.x) * (T)scale;
        r.x[1] = (T)unpack16<CK>(u.y) * (T)scale;
    }
}

// The six update coefficients of a vector of cells (x, y, z of alpha and
// beta).
template <typename T, int VK>
struct CoefV {
    Vt<T, VK> ax, ay, az, bx, by, bz;
};

template <typename T, int CK, int VK>
__device__ __forceinline__ void load_coef_v(CoefV<T, VK>& c, const StencilArgs<T>& p, int side, long long o) {
    const long long vol = p.g.vol;
    const T* a = side == 0 ? p.aE : p.aH;
    const T* b = side == 0 ? p.bE : p.bH;
    const unsigned short* qa = p.cq[2 * side];
    const unsigned short* qb = p.cq[2 * side + 1];
    const float* s = p.cs + 8 * side;
    ldg_c<T, CK, VK>(c.ax, a, qa, s[0], o);
    ldg_c<T, CK, VK>(c.ay, a, qa, s[1], vol + o);
    ldg_c<T, CK, VK>(c.az, a, qa, s[2], 2 * vol + o);
    ldg_c<T, CK, VK>(c.bx, b, qb, s[4], o);
    ldg_c<T, CK, VK>(c.by, b, qb, s[5], vol + o);
    ldg_c<T, CK, VK>(c.bz, b, qb, s[6], 2 * vol + o);
}

// E update inputs of a vector: own E and H, H one row down (j-1), and the
// single H entries just before the vector (k-1 of its first cell).
template <typename T, int VK>
struct EFldV {
    Vt<T, VK> ex, ey, ez, hx, hy, hz, hz_jm, hx_jm;
    T hy_before, hx_before;
};

// H update inputs: own H and E, E one row up (j+1), and the single E
// entries just after the vector (k+1 of its last cell).
template <typename T, int VK>
struct HFldV {
    Vt<T, VK> hx, hy, hz, ex, ey, ez, ez_jp, ex_jp;
    T ey_after, ex_after;
};

template <typename T, int VK>
__device__ __forceinline__ void load_efld_v(EFldV<T, VK>& q, const T* E, const T* __restrict__ H, long long o,
                                            long long vol, long long sj, bool edge_lane) {
    ld_v<T, VK>(q.ex, E + o);
    ld_v<T, VK>(q.ey, E + vol + o);
    ld_v<T, VK>(q.ez, E + 2 * vol + o);
    ldg_v<T, VK>(q.hx, H + o);
    ldg_v<T, VK>(q.hy, H + vol + o);
    ldg_v<T, VK>(q.hz, H + 2 * vol + o);
    ldg_v<T, VK>(q.hz_jm, H + 2 * vol + o - sj);
    ldg_v<T, VK>(q.hx_jm, H + o - sj);
    q.hy_before = edge_lane ? __ldg(H + vol + o - 1) : T(0);
    q.hx_before = edge_lane ? __ldg(H + o - 1) : T(0);
}

template <typename T, int VK>
__device__ __forceinline__ void load_hfld_v(HFldV<T, VK>& q, const T* H, const T* __restrict__ E, long long o,
                                            long long vol, long long sj, bool edge_lane) {
    ld_v<T, VK>(q.hx, H + o);
    ld_v<T, VK>(q.hy, H + vol + o);
    ld_v<T, VK>(q.hz, H + 2 * vol + o);
    ldg_v<T, VK>(q.ex, E + o);
    ldg_v<T, VK>(q.ey, E + vol + o);
    ldg_v<T, VK>(q.ez, E + 2 * vol + o);
    ldg_v<T, VK>(q.ez_jp, E + 2 * vol + o + sj);
    ldg_v<T, VK>(q.ex_jp, E + o + sj);
    q.ey_after = edge_lane ? __ldg(E + vol + o + VK) : T(0);
    q.ex_after = edge_lane ? __ldg(E + o + VK) : T(0);
}

__device__ __forceinline__ long long slab_index_v(const FaceDev& f, int l, int i, int j, int k) {
    const int a = (f.axis == 0) ? l : i;
    const int b = (f.axis == 1) ? l : j;
    const int c = (f.axis == 2) ? l : k;
    return ((long long)a * f.dJ + b) * f.pk + c;
}

// Faces (bit q = p.f[q]) whose slab a thread's cells can meet: y faces by
// the row, z faces by the vector's k range [k0, k1].
template <typename T>
__device__ __forceinline__ unsigned faces_yz(const StencilArgs<T>& p, int j, int k0, int k1) {
    unsigned m = 0;
    for (int q = 0; q < p.nfaces; ++q) {
        const FaceDev& f = p.f[q];
        if (f.axis == 1 && (unsigned)(j - f.lo) < (unsigned)f.n) m |= 1u << q;
        if (f.axis == 2 && k1 >= f.lo && k0 < f.lo + f.n) m |= 1u << q;
    }
    return m;
}

template <typename T>
__device__ __forceinline__ unsigned faces_x(const StencilArgs<T>& p, int i) {
    unsigned m = 0;
    for (int q = 0; q < p.nfaces; ++q) {
        const FaceDev& f = p.f[q];
        if (f.axis == 0 && (unsigned)(i - f.lo) < (unsigned)f.n) m |= 1u << q;
    }
    return m;
}

// CPML part of the E update of one cell (cpml.py:343-430): psi recursion
// on the faces in `mask` that contain the cell, and the correction of the
// two transverse components.  d?[axis] are the cell's curl differences
// along that axis (first, second auxiliary component).
template <typename T>
__device__ __forceinline__ void cpml_E_cell(const StencilArgs<T>& p, unsigned mask, int b, int i, int j, int k,
                                            const T (&d1)[3], const T (&d2)[3], T bx, T by, T bz, T& ex, T& ey,
                                            T& ez) {
    while (mask) {
        const int q = __ffs(mask) - 1;
        mask &= mask - 1;
        const FaceDev& f = p.f[q];
        const int coord = (f.axis == 0) ? i : ((f.axis == 1) ? j : k);
        const int l = coord - f.lo;
        if ((unsigned)l >= (unsigned)f.n) continue;
        const long long s = slab_index_v(f, l, i, j, k);
        const T* bcc = static_cast<const T*>(f.bcc);
        const T cb = bcc[l], cc = bcc[f.n + l], cck = bcc[2 * f.n + l];
        T* psi = static_cast<T*>(f.psi) + (long long)b * 4 * f.slab;
        const T e1 = f.axis == 0 ? d1[0] : (f.axis == 1 ? d1[1] : d1[2]);
        const T e2 = f.axis == 0 ? d2[0] : (f.axis == 1 ? d2[1] : d2[2]);
        T p1 = psi[s] * cb;
        p1 = p1 + cc * e1;
        if (!f.air[s]) p1 = T(0);
        psi[s] = p1;
        T p2 = psi[f.slab + s] * cb;
        p2 = p2 + cc * e2;
        if (!f.air[f.slab + s]) p2 = T(0);
        psi[f.slab + s] = p2;
        if (f.axis == 0) {
            ey = ey + by * (cck * e1 + p1);
            ez = ez - bz * (cck * e2 + p2);
        } else if (f.axis == 1) {
            ex = ex - bx * (cck * e1 + p1);
            ez = ez + bz * (cck * e2 + p2);
        } else {
            ex = ex + bx * (cck * e1 + p1);
            ey = ey - by * (cck * e2 + p2);
        }
    }
}

// CPML part of the H update of one cell (cpml.py:432-516).
template <typename T>
__device__ __forceinline__ void cpml_H_cell(const StencilArgs<T>& p, unsigned mask, int b, int i, int j, int k,
                                            const T (&d1)[3], const T (&d2)[3], T bx, T by, T bz, T& hx, T& hy,
                                            T& hz) {
    while (mask) {
        const int q = __ffs(mask) - 1;
        mask &= mask - 1;
        const FaceDev& f = p.f[q];
        const int coord = (f.axis == 0) ? i : ((f.axis == 1) ? j : k);
        const int l = coord - f.lo;
        if ((unsigned)l >= (unsigned)f.n) continue;
        const long long s = slab_index_v(f, l, i, j, k);
        const T* bcc = static_cast<const T*>(f.bcc);
        const T cb = bcc[l], cc = bcc[f.n + l], cck = bcc[2 * f.n + l];
        T* psi = static_cast<T*>(f.psi) + (long long)b * 4 * f.slab;
        const T e1 = f.axis == 0 ? d1[0] : (f.axis == 1 ? d1[1] : d1[2]);
        const T e2 = f.axis == 0 ? d2[0] : (f.axis == 1 ? d2[1] : d2[2]);
        const long long s1 = 2 * f.slab + s, s2 = 3 * f.slab + s;
        T p1 = psi[s1] * cb;
        p1 = p1 + cc * e1;
        if (!f.air[s1]) p1 = T(0);
        psi[s1] = p1;
        T p2 = psi[s2] * cb;
        p2 = p2 + cc * e2;
        if (!f.air[s2]) p2 = T(0);
        psi[s2] = p2;
        if (f.axis == 0) {
            hy = hy - by * (cck * e1 + p1);
            hz = hz + bz * (cck * e2 + p2);
        } else if (f.axis == 1) {
            hx = hx + bx * (cck * e1 + p1);
            hz = hz - bz * (cck * e2 + p2);
        } else {
            hx = hx - bx * (cck * e1 + p1);
            hy = hy + by * (cck * e2 + p2);
        }
    }
}

constexpr unsigned kFull = 0xffffffffu;

// Work item of a thread: vector vq of the plane (clamped to the last vector
// for the idle lanes of the last warp, which load but never store).
struct VecItem {
    bool live;
    int j, k0;
    long long e0;
};

template <typename T, int VK>
__device__ __forceinline__ VecItem vec_item(const Geom& g, int B) {
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int warps = blockDim.x >> 5;
    const long long nvec = (long long)(g.ny + 1) * g.nkp / VK;
    const long long vq = ((long long)blockIdx.x * (warps / B) + w / B) * 32 + lane;
    VecItem it;
    it.live = vq < nvec;
    it.e0 = (it.live ? vq : nvec - 1) * VK;
    it.j = (int)(it.e0 / g.nkp);
    it.k0 = (int)(it.e0 - (long long)it.j * g.nkp);
    return it;
}

template <typename T, int CK, int VK, int MINB>
__global__ void __launch_bounds__(256, MINB) k_update_E_vec(const StencilArgs<T> p) {
    const Geom& g = p.g;
    const int B = p.B;
    const int b = (threadIdx.x >> 5) % B;
    const int lane = threadIdx.x & 31;
    const VecItem it = vec_item<T, VK>(g, B);
    // the warp's first vector is beyond the plane: no lane has work
    if (__all_sync(kFull, !it.live)) return;
    const int j = it.j, k0 = it.k0;
    const int nstore = it.live ? max(0, min(VK, g.nz + 1 - k0)) : 0;
    const int i0 = blockIdx.z * p.ichunk;
    const int i1 = min(i0 + p.ichunk, g.nx + 1);
    const long long vol = g.vol, si = g.si, sj = g.sj, fs = 3 * vol;
    T* E = p.e + b * fs;
    const T* __restrict__ H = p.h + b * fs;
    const unsigned myz = (nstore > 0) ? faces_yz(p, j, k0, k0 + nstore - 1) : 0u;
    long long o = (long long)(i0 + 2) * si + it.e0;
    Vt<T, VK> hz_im, hy_im;
    ldg_v<T, VK>(hz_im, H + 2 * vol + o - si);
    ldg_v<T, VK>(hy_im, H + vol + o - si);
    CoefV<T, VK> cc, cn;
    EFldV<T, VK> fc, fn;
    load_coef_v<T, CK, VK>(cc, p, 0, o);
    load_efld_v<T, VK>(fc, E, H, o, vol, sj, lane == 0);
    for (int i = i0; i < i1; ++i) {
        if (i + 1 < i1) {
            load_coef_v<T, CK, VK>(cn, p, 0, o + si);
            load_efld_v<T, VK>(fn, E, H, o + si, vol, sj, lane == 0);
        }
        // k-1 entries: the previous lane's last entry, or the loaded one
        const T hy_prev = __shfl_up_sync(kFull, fc.hy.x[VK - 1], 1);
        const T hx_prev = __shfl_up_sync(kFull, fc.hx.x[VK - 1], 1);
        const unsigned mask = nstore > 0 ? (myz | faces_x(p, i)) : 0u;
        Vt<T, VK> ex, ey, ez;
#pragma unroll
        for (int e = 0; e < VK; ++e) {
            const T hy_km = e > 0 ? fc.hy.x[e - 1] : (lane == 0 ? fc.hy_before : hy_prev);
            const T hx_km = e > 0 ? fc.hx.x[e - 1] : (lane == 0 ? fc.hx_before : hx_prev);
            const T hx = fc.hx.x[e], hy = fc.hy.x[e], hz = fc.hz.x[e];
            const T cx = ((hz - fc.hz_jm.x[e]) - hy) + hy_km;
            const T cy = ((hx - hx_km) - hz) + hz_im.x[e];
            const T cz = ((hy - hy_im.x[e]) - hx) + fc.hx_jm.x[e];
            ex.x[e] = cc.ax.x[e] * fc.ex.x[e] + cc.bx.x[e] * cx;
            ey.x[e] = cc.ay.x[e] * fc.ey.x[e] + cc.by.x[e] * cy;
            ez.x[e] = cc.az.x[e] * fc.ez.x[e] + cc.bz.x[e] * cz;
            if (mask && e < nstore) {
                const T d1[3] = {hz - hz_im.x[e], hz - fc.hz_jm.x[e], hy - hy_km};
                const T d2[3] = {hy - hy_im.x[e], hx - fc.hx_jm.x[e], hx - hx_km};
                cpml_E_cell(p, mask, b, i, j, k0 + e, d1, d2, cc.bx.x[e], cc.by.x[e], cc.bz.x[e], ex.x[e], ey.x[e],
                            ez.x[e]);
            }
            hz_im.x[e] = hz;
            hy_im.x[e] = hy;
        }
        st_v_n<T, VK>(E + o, ex, nstore);
        st_v_n<T, VK>(E + vol + o, ey, nstore);
        st_v_n<T, VK>(E + 2 * vol + o, ez, nstore);
        cc = cn;
        fc = fn;
        o += si;
    }
}

template <typename T, int CK, int VK, int MINB>
__global__ void __launch_bounds__(256, MINB) k_update_H_vec(const StencilArgs<T> p) {
    const Geom& g = p.g;
    const int B = p.B;
    const int b = (threadIdx.x >> 5) % B;
    const int lane = threadIdx.x & 31;
    const VecItem it = vec_item<T, VK>(g, B);
    if (__all_sync(kFull, !it.live)) return;
    const int j = it.j, k0 = it.k0;
    const int nstore = it.live ? max(0, min(VK, g.nz + 1 - k0)) : 0;
    const int i0 = blockIdx.z * p.ichunk;
    const int i1 = min(i0 + p.ichunk, g.nx + 1);
    const long long vol = g.vol, si = g.si, sj = g.sj, fs = 3 * vol;
    T* H = p.h + b * fs;
    const T* __restrict__ E = p.e + b * fs;
    const unsigned myz = (nstore > 0) ? faces_yz(p, j, k0, k0 + nstore - 1) : 0u;
    // march down: the x-neighbours (E at i+1) of the first plane
    long long o = (long long)(i1 - 1 + 2) * si + it.e0;
    Vt<T, VK> ez_ip, ey_ip;
    ldg_v<T, VK>(ez_ip, E + 2 * vol + o + si);
    ldg_v<T, VK>(ey_ip, E + vol + o + si);
    CoefV<T, VK> cc, cn;
    HFldV<T, VK> fc, fn;
    load_coef_v<T, CK, VK>(cc, p, 1, o);
    load_hfld_v<T, VK>(fc, H, E, o, vol, sj, lane == 31);
    for (int i = i1 - 1; i >= i0; --i) {
        if (i - 1 >= i0) {
            load_coef_v<T, CK, VK>(cn, p, 1, o - si);
            load_hfld_v<T, VK>(fn, H, E, o - si, vol, sj, lane == 31);
        }
        // k+1 entries: the next lane's first entry, or the loaded one
        const T ey_next = __shfl_down_sync(kFull, fc.ey.x[0], 1);
        const T ex_next = __shfl_down_sync(kFull, fc.ex.x[0], 1);
        const unsigned mask = nstore > 0 ? (myz | faces_x(p, i)) : 0u;
        Vt<T, VK> hx, hy, hz;
#pragma unroll
        for (int e = 0; e < VK; ++e) {
            const T ey_kp = e < VK - 1 ? fc.ey.x[e + 1] : (lane == 31 ? fc.ey_after : ey_next);
            const T ex_kp = e < VK - 1 ? fc.ex.x[e + 1] : (lane == 31 ? fc.ex_after : ex_next);
            const T ex = fc.ex.x[e], ey = fc.ey.x[e], ez = fc.ez.x[e];
            const T cx = ((fc.ez_jp.x[e] - ez) - ey_kp) + ey;
            const T cy = ((ex_kp - ex) - ez_ip.x[e]) + ez;
            const T cz = ((ey_ip.x[e] - ey) - fc.ex_jp.x[e]) + ex;
            hx.x[e] = cc.ax.x[e] * fc.hx.x[e] - cc.bx.x[e] * cx;
            hy.x[e] = cc.ay.x[e] * fc.hy.x[e] - cc.by.x[e] * cy;
            hz.x[e] = cc.az.x[e] * fc.hz.x[e] - cc.bz.x[e] * cz;
            if (mask && e < nstore) {
                const T d1[3] = {ez_ip.x[e] - ez, fc.ez_jp.x[e] - ez, ey_kp - ey};
                const T d2[3] = {ey_ip.x[e] - ey, fc.ex_jp.x[e] - ex, ex_kp - ex};
                cpml_H_cell(p, mask, b, i, j, k0 + e, d1, d2, cc.bx.x[e], cc.by.x[e], cc.bz.x[e], hx.x[e], hy.x[e],
                            hz.x[e]);
            }
            ez_ip.x[e] = ez;
            ey_ip.x[e] = ey;
        }
        st_v_n<T, VK>(H + o, hx, nstore);
        st_v_n<T, VK>(H + vol + o, hy, nstore);
        st_v_n<T, VK>(H + 2 * vol + o, hz, nstore);
        cc = cn;
        fc = fn;
        o -= si;
    }
}

// Variants (vector width, minimum resident CTAs of 256 threads per SM,
// which caps the registers): 0 = (4, 1), 1 = (4, 2), 2 = (2, 2), 3 = (2, 3)
// in float32; float64 uses width 2 with the same caps.
constexpr int kVecVariants = 4;

int vec_warps(int) { return 8; }

template <typename T, int CK, int VK, int MINB>
void occ_one(int& a, int& c) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_update_E_vec<T, CK, VK, MINB>, 256, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c, k_update_H_vec<T, CK, VK, MINB>, 256, 0);
}

template <typename T, int CK, int VK, int MINB>
void launch_one(const StencilArgs<T>& a, dim3 grid, int which, cudaStream_t s) {
    if (which == 0)
        k_update_E_vec<T, CK, VK, MINB><<<grid, 256, 0, s>>>(a);
    else
        k_update_H_vec<T, CK, VK, MINB><<<grid, 256, 0, s>>>(a);
}

// Native coefficients: every variant; 16-bit coefficients: variant 0.
template <typename T, typename F>
void dispatch(int variant, int coef_kind, F&& f) {
    constexpr int W = sizeof(T) == 4 ? 4 : 2;
    if (coef_kind == kCoefF16) return f.template run<kCoefF16, W, 1>();
    if (coef_kind == kCoefBF16) return f.template run<kCoefBF16, W, 1>();
    switch (variant) {
        case 1: return f.template run<kCoefNative, W, 2>();
        case 2: return f.template run<kCoefNative, 2, 2>();
        case 3: return f.template run<kCoefNative, 2, 3>();
        default: return f.template run<kCoefNative, W, 1>();
    }
}

template <typename T>
struct OccF {
    int a = 0, c = 0;
    template <int CK, int VK, int MINB>
    void run() { occ_one<T, CK, VK, MINB>(a, c); }
};

template <typename T>
struct LaunchF {
    const StencilArgs<T>& a;
    dim3 grid;
    int which;
    cudaStream_t s;
    template <int CK, int VK, int MINB>
    void run() { launch_one<T, CK, VK, MINB>(a, grid, which, s); }
};

}  // namespace

int vec_width_of(int prec, int variant) { return (prec == 4 && variant < 2) ? 4 : 2; }

template <typename T>
int vec_occupancy(int variant, int coef_kind) {
    OccF<T> f;
    dispatch<T>(variant, coef_kind, f);
    const int m = f.a < f.c ? f.a : f.c;
    return m < 1 ? 1 : m;
}
template int vec_occupancy<float>(int, int);
template int vec_occupancy<double>(int, int);

StreamPlan plan_vec(const Geom& g, int sm_count, int ctas_per_sm, int B, int vk) {
    StreamPlan s{};
    s.block_y = vec_warps(B);
    const long long nvec = (long long)(g.ny + 1) * g.nkp / vk;
    const long long per_cta = 32LL * (s.block_y / B);
    const int bx = (int)((nvec + per_cta - 1) / per_cta);
    const int nplanes = g.nx + 1;
    const int per_wave = sm_count * ctas_per_sm;
    double best = -1.0;
    int best_chunk = nplanes;
    for (int ichunk = nplanes; ichunk >= 4; --ichunk) {
        const int nch = (nplanes + ichunk - 1) / ichunk;
        const double waves = (double)bx * nch / per_wave;
        const double eff = waves / (double)((long long)(waves + 0.999999));
        const double score = eff - 0.5 / ichunk;
        if (score > best) {
            best = score;
            best_chunk = ichunk;
        }
    }
    s.ichunk = best_chunk;
    s.grid_x = bx;
    s.grid_y = 1;
    s.grid_z = (nplanes + best_chunk - 1) / best_chunk;
    return s;
}

template <typename T>
void launch_vec_half(StencilArgs<T> a, const StreamPlan& sp, int variant, int which, cudaStream_t s) {
    a.ichunk = sp.ichunk;
    LaunchF<T> f{a, dim3(sp.grid_x, sp.grid_y, sp.grid_z), which, s};
    dispatch<T>(variant, a.coef_kind, f);
}
template void launch_vec_half<float>(StencilArgs<float>, const StreamPlan&, int, int, cudaStream_t);
template void launch_vec_half<double>(StencilArgs<double>, const StreamPlan&, int, int, cudaStream_t);

}  // namespace fitb
