// Software-pipelined leapfrog curl updates, batched over field sets.
//
// Same arithmetic and in-thread order as stencil.cu (reference:
// numba_kernels.py:36-127, cpml.py:343-516).  One thread owns a (j, k)
// column of one field set and marches over a chunk of i planes.  Per plane
// it loads the six update coefficients of its cell, the cell's fields and
// its four in-plane neighbours; the next plane's loads are issued before the
// current plane is computed, so a thread always has a full plane of
// independent loads in flight while it does arithmetic (a deeper in-register
// queue, and a per-thread loop over field sets, both measured slower: the
// extra registers cost more warps than they gain).  The x-neighbours come
// from registers: the E update marches up in i (it needs H at i-1, the
// previous plane's values), the H update marches down (it needs E at i+1).
// Batched form (all port x mode excitations of one mesh advancing
// together): the B field sets of a cell run in B warps of the same CTA.
#include "fitb_common.cuh"
#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace fitb {

namespace {

constexpr int kSX = 32;
constexpr int kSY = 8;

template <typename T>
struct Coef {
    T ax, ay, az, bx, by, bz;
};

// Field values of one cell for the E update: own E and H, H neighbours at
// j-1 (Hz, Hx) and k-1 (Hy, Hx).
template <typename T>
struct EFld {
    T ex, ey, ez, hx, hy, hz, hz_jm, hx_jm, hy_km, hx_km;
};

// For the H update: own H and E, E neighbours at j+1 (Ez, Ex), k+1 (Ey, Ex).
template <typename T>
struct HFld {
    T hx, hy, hz, ex, ey, ez, ez_jp, ex_jp, ey_kp, ex_kp;
};

__device__ __forceinline__ long long slab_index_s(const FaceDev& f, int l, int i, int j, int k) {
    const int a = (f.axis == 0) ? l : i;
    const int b = (f.axis == 1) ? l : j;
    const int c = (f.axis == 2) ? l : k;
    return ((long long)a * f.dJ + b) * f.pk + c;
}

template <typename T>
__device__ __forceinline__ void load_coef(Coef<T>& q, const T* __restrict__ a, const T* __restrict__ b, long long o,
                                          long long vol) {
    q.ax = __ldg(a + o);
    q.ay = __ldg(a + vol + o);
    q.az = __ldg(a + 2 * vol + o);
    q.bx = __ldg(b + o);
    q.by = __ldg(b + vol + o);
    q.bz = __ldg(b + 2 * vol + o);
}

template <int CK>
__device__ __forceinline__ float unpack16(unsigned short u) {
    if constexpr (CK == kCoefF16)
        return __half2float(__ushort_as_half(u));
    else
        return __bfloat162float(__ushort_as_bfloat16(u));
}

// Coefficients of one cell in the handle's storage: native, or 16-bit with a
// per-array scale (side 0: alpha_E / beta_E, side 1: alpha_H / beta_H).
template <typename T, int CK>
__device__ __forceinline__ void load_coef_k(Coef<T>& q, const StencilArgs<T>& p, int side, const T* __restrict__ a,
                                            const T* __restrict__ b, long long o, long long vol) {
    if constexpr (CK == kCoefNative) {
        load_coef(q, a, b, o, vol);
    } else {
        const unsigned short* __restrict__ qa = p.cq[2 * side];
        const unsigned short* __restrict__ qb = p.cq[2 * side + 1];
        const float* s = p.cs + 8 * side;
        q.ax = (T)unpack16<CK>(__ldg(qa + o)) * (T)s[0];
        q.ay = (T)unpack16<CK>(__ldg(qa + vol + o)) * (T)s[1];
        q.az = (T)unpack16<CK>(__ldg(qa + 2 * vol + o)) * (T)s[2];
        q.bx = (T)unpack16<CK>(__ldg(qb + o)) * (T)s[4];
        q.by = (T)unpack16<CK>(__ldg(qb + vol + o)) * (T)s[5];
        q.bz = (T)unpack16<CK>(__ldg(qb + 2 * vol + o)) * (T)s[6];
    }
}

template <typename T>
__device__ __forceinline__ void load_efld(EFld<T>& q, const T* E, const T* __restrict__ H, long long o, long long vol,
                                          long long sj) {
    q.ex = E[o];
    q.ey = E[vol + o];
    q.ez = E[2 * vol + o];
    q.hx = __ldg(H + o);
    q.hy = __ldg(H + vol + o);
    q.hz = __ldg(H + 2 * vol + o);
    q.hz_jm = __ldg(H + 2 * vol + o - sj);
    q.hx_jm = __ldg(H + o - sj);
    q.hy_km = __ldg(H + vol + o - 1);
    q.hx_km = __ldg(H + o - 1);
}

template <typename T>
__device__ __forceinline__ void load_hfld(HFld<T>& q, const T* H, const T* __restrict__ E, long long o, long long vol,
                                          long long sj) {
    q.hx = H[o];
    q.hy = H[vol + o];
    q.hz = H[2 * vol + o];
    q.ex = __ldg(E + o);
    q.ey = __ldg(E + vol + o);
    q.ez = __ldg(E + 2 * vol + o);
    q.ez_jp = __ldg(E + 2 * vol + o + sj);
    q.ex_jp = __ldg(E + o + sj);
    q.ey_kp = __ldg(E + vol + o + 1);
    q.ex_kp = __ldg(E + o + 1);
}

template <typename T>
__device__ __forceinline__ void compute_E(const StencilArgs<T>& p, const Coef<T>& c, const EFld<T>& cur, T& hz_im,
                                          T& hy_im, int b, int i, int j, int k, long long o, long long vol,
                                          unsigned mask) {
    T* __restrict__ E = p.e + (long long)b * 3 * vol;
    const T cx = ((cur.hz - cur.hz_jm) - cur.hy) + cur.hy_km;
    const T cy = ((cur.hx - cur.hx_km) - cur.hz) + hz_im;
    const T cz = ((cur.hy - hy_im) - cur.hx) + cur.hx_jm;
    T ex = c.ax * cur.ex + c.bx * cx;
    T ey = c.ay * cur.ey + c.by * cy;
    T ez = c.az * cur.ez + c.bz * cz;
    while (mask) {
        const int fi = __ffs(mask) - 1;
        mask &= mask - 1;
        const FaceDev& f = p.f[fi];
        const int coord = (f.axis == 0) ? i : ((f.axis == 1) ? j : k);
        const int l = coord - f.lo;
        const long long s = slab_index_s(f, l, i, j, k);
        const T* bcc = static_cast<const T*>(f.bcc);
        const T cb = bcc[l], cc = bcc[f.n + l], cck = bcc[2 * f.n + l];
        T* psi = static_cast<T*>(f.psi) + (long long)b * 4 * f.slab;
        T d1, d2;
        if (f.axis == 0) {
            d1 = cur.hz - hz_im;
            d2 = cur.hy - hy_im;
        } else if (f.axis == 1) {
            d1 = cur.hz - cur.hz_jm;
            d2 = cur.hx - cur.hx_jm;
        } else {
            d1 = cur.hy - cur.hy_km;
            d2 = cur.hx - cur.hx_km;
        }
        T p1 = psi[s] * cb;
        p1 = p1 + cc * d1;
        if (!f.air[s]) p1 = T(0);
        psi[s] = p1;
        T p2 = psi[f.slab + s] * cb;
        p2 = p2 + cc * d2;
        if (!f.air[f.slab + s]) p2 = T(0);
        psi[f.slab + s] = p2;
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
    E[o] = ex;
    E[vol + o] = ey;
    E[2 * vol + o] = ez;
    hz_im = cur.hz;
    hy_im = cur.hy;
}

template <typename T>
__device__ __forceinline__ void compute_H(const StencilArgs<T>& p, const Coef<T>& c, const HFld<T>& cur, T& ez_ip,
                                          T& ey_ip, int b, int i, int j, int k, long long o, long long vol,
                                          unsigned mask) {
    T* __restrict__ H = p.h + (long long)b * 3 * vol;
    const T cx = ((cur.ez_jp - cur.ez) - cur.ey_kp) + cur.ey;
    const T cy = ((cur.ex_kp - cur.ex) - ez_ip) + cur.ez;
    const T cz = ((ey_ip - cur.ey) - cur.ex_jp) + cur.ex;
    T hx = c.ax * cur.hx - c.bx * cx;
    T hy = c.ay * cur.hy - c.by * cy;
    T hz = c.az * cur.hz - c.bz * cz;
    while (mask) {
        const int fi = __ffs(mask) - 1;
        mask &= mask - 1;
        const FaceDev& f = p.f[fi];
        const int coord = (f.axis == 0) ? i : ((f.axis == 1) ? j : k);
        const int l = coord - f.lo;
        const long long s = slab_index_s(f, l, i, j, k);
        const T* bcc = static_cast<const T*>(f.bcc);
        const T cb = bcc[l], cc = bcc[f.n + l], cck = bcc[2 * f.n + l];
        T* psi = static_cast<T*>(f.psi) + (long long)b * 4 * f.slab;
        T d1, d2;
        if (f.axis == 0) {
            d1 = ez_ip - cur.ez;
            d2 = ey_ip - cur.ey;
        } else if (f.axis == 1) {
            d1 = cur.ez_jp - cur.ez;
            d2 = cur.ex_jp - cur.ex;
        } else {
            d1 = cur.ey_kp - cur.ey;
            d2 = cur.ex_kp - cur.ex;
        }
        const long long s1 = 2 * f.slab + s, s2 = 3 * f.slab + s;
        T p1 = psi[s1] * cb;
        p1 = p1 + cc * d1;
        if (!f.air[s1]) p1 = T(0);
        psi[s1] = p1;
        T p2 = psi[s2] * cb;
        p2 = p2 + cc * d2;
        if (!f.air[s2]) p2 = T(0);
        psi[s2] = p2;
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
    H[o] = hx;
    H[vol + o] = hy;
    H[2 * vol + o] = hz;
    ez_ip = cur.ez;
    ey_ip = cur.ey;
}

// Faces (bit q = p.f[q]) that contain cell column (j, k): the y and z faces,
// fixed for a thread; the x faces that contain plane i.
template <typename T>
__device__ __forceinline__ unsigned faces_jk(const StencilArgs<T>& p, int j, int k) {
    unsigned m = 0;
    for (int q = 0; q < p.nfaces; ++q) {
        const FaceDev& f = p.f[q];
        const int c = f.axis == 1 ? j : k;
        if (f.axis != 0 && (unsigned)(c - f.lo) < (unsigned)f.n) m |= 1u << q;
    }
    return m;
}

template <typename T>
__device__ __forceinline__ unsigned faces_i(const StencilArgs<T>& p, int i) {
    unsigned m = 0;
    for (int q = 0; q < p.nfaces; ++q) {
        const FaceDev& f = p.f[q];
        if (f.axis == 0 && (unsigned)(i - f.lo) < (unsigned)f.n) m |= 1u << q;
    }
    return m;
}

// Field sets map to the warps of one CTA: warp row ty handles field set
// b = ty % B of grid row j = blockIdx.y * rows + ty / B.  Each thread runs the
// single-field-set pipeline; the B warps that share a cell load the same
// coefficients, which the first of them brings from HBM and the others find
// in L1/L2, so the coefficients cross HBM once per cell for all field sets
// while every thread keeps a full plane of loads in flight.
// MAXT / MINB: launch bounds of the register-capped variants (see
// stream_dispatch below).
template <typename T, int CK, int MAXT = 512, int MINB = 1>
__global__ void __launch_bounds__(MAXT, MINB) k_update_E_stream(const StencilArgs<T> p) {
    const Geom& g = p.g;
    const int B = p.B;
    const int b = threadIdx.y % B;
    const int k = blockIdx.x * kSX + threadIdx.x;
    const int j = blockIdx.y * (blockDim.y / B) + threadIdx.y / B;
    if (k > g.nz || j > g.ny) return;
    const int i0 = blockIdx.z * p.ichunk;
    const int i1 = min(i0 + p.ichunk, g.nx + 1);
    const long long vol = g.vol, si = g.si, sj = g.sj, fs = 3 * vol;
    const T* __restrict__ aE = p.aE;
    const T* __restrict__ bE = p.bE;
    const T* E = p.e + b * fs;
    const T* __restrict__ H = p.h + b * fs;
    const unsigned mjk = faces_jk(p, j, k);
    long long o = pidx(g, i0, j, k);
    T hz_im = __ldg(H + 2 * vol + o - si);
    T hy_im = __ldg(H + vol + o - si);
    Coef<T> cc, cn;
    EFld<T> fc, fn;
    load_coef_k<T, CK>(cc, p, 0, aE, bE, o, vol);
    load_efld(fc, E, H, o, vol, sj);
    for (int i = i0; i < i1; ++i) {
        if (i + 1 < i1) {
            load_coef_k<T, CK>(cn, p, 0, aE, bE, o + si, vol);
            load_efld(fn, E, H, o + si, vol, sj);
        }
        compute_E(p, cc, fc, hz_im, hy_im, b, i, j, k, o, vol, mjk | faces_i(p, i));
        cc = cn;
        fc = fn;
        o += si;
    }
}

template <typename T, int CK, int MAXT = 512, int MINB = 1>
__global__ void __launch_bounds__(MAXT, MINB) k_update_H_stream(const StencilArgs<T> p) {
    const Geom& g = p.g;
    const int B = p.B;
    const int b = threadIdx.y % B;
    const int k = blockIdx.x * kSX + threadIdx.x;
    const int j = blockIdx.y * (blockDim.y / B) + threadIdx.y / B;
    if (k > g.nz || j > g.ny) return;
    const int i0 = blockIdx.z * p.ichunk;
    const int i1 = min(i0 + p.ichunk, g.nx + 1);
    const long long vol = g.vol, si = g.si, sj = g.sj, fs = 3 * vol;
    const T* __restrict__ aH = p.aH;
    const T* __restrict__ bH = p.bH;
    const T* H = p.h + b * fs;
    const T* __restrict__ E = p.e + b * fs;
    // march down: the x-neighbours (E at i+1) of the first plane
    const unsigned mjk = faces_jk(p, j, k);
    long long o = pidx(g, i1 - 1, j, k);
    T ez_ip = __ldg(E + 2 * vol + o + si);
    T ey_ip = __ldg(E + vol + o + si);
    Coef<T> cc, cn;
    HFld<T> fc, fn;
    load_coef_k<T, CK>(cc, p, 1, aH, bH, o, vol);
    load_hfld(fc, H, E, o, vol, sj);
    for (int i = i1 - 1; i >= i0; --i) {
        if (i - 1 >= i0) {
            load_coef_k<T, CK>(cn, p, 1, aH, bH, o - si, vol);
            load_hfld(fn, H, E, o - si, vol, sj);
        }
        compute_H(p, cc, fc, ez_ip, ey_ip, b, i, j, k, o, vol, mjk | faces_i(p, i));
        cc = cn;
        fc = fn;
        o -= si;
    }
}

int block_rows_y(int B) { return B <= 8 ? 8 : B; }

// Register-capped variants of the native-coefficient kernels (more warps
// resident per SM; the kernels are DRAM-latency bound):
//   0: __launch_bounds__(512, 2): <= 64 registers (the default: four CTAs
//      of 256 per SM, no spills);
//   1: natural allocation (72-80 registers in float32, fewer CTAs);
//   2: __launch_bounds__(256, 5): <= 48 registers, blocks of 256 only;
//   3: __launch_bounds__(256, 6): <= 40 registers, blocks of 256 only.
template <typename T, typename F>
void stream_dispatch(int variant, int coef_kind, F&& f) {
    if (coef_kind == kCoefF16) return f.template run<kCoefF16, 512, 2>();
    if (coef_kind == kCoefBF16) return f.template run<kCoefBF16, 512, 2>();
    switch (variant) {
        case 1: return f.template run<kCoefNative, 512, 1>();
        case 2: return f.template run<kCoefNative, 256, 5>();
        case 3: return f.template run<kCoefNative, 256, 6>();
        default: return f.template run<kCoefNative, 512, 2>();
    }
}

template <typename T>
struct StreamOcc {
    int threads, a = 0, c = 0;
    template <int CK, int MAXT, int MINB>
    void run() {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_update_E_stream<T, CK, MAXT, MINB>, threads, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c, k_update_H_stream<T, CK, MAXT, MINB>, threads, 0);
    }
};

template <typename T>
struct StreamLaunch {
    const StencilArgs<T>& a;
    dim3 grid, block;
    int which;
    cudaStream_t s;
    template <int CK, int MAXT, int MINB>
    void run() {
        if (which == 0)
            k_update_E_stream<T, CK, MAXT, MINB><<<grid, block, 0, s>>>(a);
        else
            k_update_H_stream<T, CK, MAXT, MINB><<<grid, block, 0, s>>>(a);
    }
};

}  // namespace

bool stream_batch_supported(int B) { return B == 1 || B == 2 || B == 4 || B == 8 || B == 16; }

bool stream_variant_supported(int B, int variant) {
    return variant == 0 || variant == 1 || ((variant == 2 || variant == 3) && B <= 8);
}

template <typename T>
int stream_occupancy(int B, int coef_kind, int variant) {
    StreamOcc<T> f{kSX * block_rows_y(B)};
    stream_dispatch<T>(variant, coef_kind, f);
    const int m = f.a < f.c ? f.a : f.c;
    return m < 1 ? 1 : m;
}
template int stream_occupancy<float>(int, int, int);
template int stream_occupancy<double>(int, int, int);

StreamPlan plan_stream(const Geom& g, int sm_count, int ctas_per_sm, int B) {
    StreamPlan s{};
    s.block_y = block_rows_y(B);
    const int rows = s.block_y / B;
    const int bx = (g.nz + 1 + kSX - 1) / kSX, by = (g.ny + 1 + rows - 1) / rows;
    const int nplanes = g.nx + 1;
    const int per_wave = sm_count * ctas_per_sm;
    // chunks of 12-32 planes: longer ones leave few CTAs that all sweep the
    // same planes in step with one plane of loads in flight each (measured:
    // a single 257-plane wave at 256^3 and B = 2 runs 1.6x slower than
    // chunks of 16); among those, prefer long chunks (fewer re-loaded
    // boundary planes) unless the wave tail costs more than a few percent
    double best = -1.0;
    int best_chunk = std::min(nplanes, 16);
    for (int ichunk = std::min(nplanes, 32); ichunk >= std::min(nplanes, 12); --ichunk) {
        const int nch = (nplanes + ichunk - 1) / ichunk;
        const double waves = (double)bx * by * nch / per_wave;
        const double eff = waves / (double)((long long)(waves + 0.999999));
        const double score = eff - 0.5 / ichunk;
        if (score > best) {
            best = score;
            best_chunk = ichunk;
        }
    }
    s.ichunk = best_chunk;
    s.grid_x = bx;
    s.grid_y = by;
    s.grid_z = (nplanes + best_chunk - 1) / best_chunk;
    return s;
}

template <typename T>
void launch_stream_half(StencilArgs<T> a, const StreamPlan& sp, int variant, int which, cudaStream_t s) {
    a.ichunk = sp.ichunk;
    StreamLaunch<T> f{a, dim3(sp.grid_x, sp.grid_y, sp.grid_z), dim3(kSX, sp.block_y, 1), which, s};
    stream_dispatch<T>(variant, a.coef_kind, f);
}

template void launch_stream_half<float>(StencilArgs<float>, const StreamPlan&, int, int, cudaStream_t);
template void launch_stream_half<double>(StencilArgs<double>, const StreamPlan&, int, int, cudaStream_t);

}  // namespace fitb

namespace fitb {
namespace {

template <typename T, int CK>
__global__ void k_compact(const T* __restrict__ src, unsigned short* __restrict__ dst, long long n, float inv_scale) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const float v = (float)src[q] * inv_scale;
        if constexpr (CK == kCoefF16)
            dst[q] = __half_as_ushort(__float2half_rn(v));
        else
            dst[q] = __bfloat16_as_ushort(__float2bfloat16_rn(v));
    }
}

}  // namespace

template <typename T>
void launch_compact(const T* src, unsigned short* dst, long long n, float inv_scale, int coef_kind, cudaStream_t s) {
    const int threads = 256;
    const long long want = (n + threads - 1) / threads;
    const int blocks = (int)(want < 148 * 16 ? want : 148 * 16);
    if (blocks < 1) return;
    if (coef_kind == kCoefF16)
        k_compact<T, kCoefF16><<<blocks, threads, 0, s>>>(src, dst, n, inv_scale);
    else
        k_compact<T, kCoefBF16><<<blocks, threads, 0, s>>>(src, dst, n, inv_scale);
}
template void launch_compact<float>(const float*, unsigned short*, long long, float, int, cudaStream_t);
template void launch_compact<double>(const double*, unsigned short*, long long, float, int, cudaStream_t);

}  // namespace fitb
