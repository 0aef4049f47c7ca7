// Software-pipelined leapfrog curl updates for one field set.
//
// Same arithmetic and in-thread order as stencil.cu (reference:
// numba_kernels.py:36-127, cpml.py:343-516).  One thread owns a (j, k)
// column and marches over a chunk of i planes; every plane's sixteen loads
// (the cell's own coefficients, fields and its four in-plane neighbours) are
// issued for plane i+1 before plane i is computed, so a thread always has a
// whole plane of independent loads in flight while it does arithmetic (two
// planes ahead measured slower: the extra registers cost more warps than
// the deeper queue gains).  The
// x-neighbours come from registers: the E update marches up in i (it needs
// H at i-1, the previous iteration's values), the H update marches down (it
// needs E at i+1).
#include "fitb_common.cuh"

namespace fitb {

namespace {

constexpr int kSX = 32;
constexpr int kSY = 8;

template <typename T>
struct EPlane {
    T ax, ay, az, bx, by, bz, ex, ey, ez, hx, hy, hz, hz_jm, hx_jm, hy_km, hx_km;
};

template <typename T>
struct HPlane {
    T ax, ay, az, bx, by, bz, hx, hy, hz, ex, ey, ez, ez_jp, ex_jp, ey_kp, ex_kp;
};

template <typename T>
__device__ __forceinline__ long long slab_index_s(const FaceDev& f, int l, int i, int j, int k) {
    const int a = (f.axis == 0) ? l : i;
    const int b = (f.axis == 1) ? l : j;
    const int c = (f.axis == 2) ? l : k;
    return ((long long)a * f.dJ + b) * f.dK + c;
}

template <typename T>
__device__ __forceinline__ void load_E_plane(EPlane<T>& q, const T* __restrict__ aE, const T* __restrict__ bE,
                                             const T* __restrict__ E, const T* __restrict__ H, long long o,
                                             long long vol, long long sj) {
    q.ax = __ldg(aE + o);
    q.ay = __ldg(aE + vol + o);
    q.az = __ldg(aE + 2 * vol + o);
    q.bx = __ldg(bE + o);
    q.by = __ldg(bE + vol + o);
    q.bz = __ldg(bE + 2 * vol + o);
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
__device__ __forceinline__ void load_H_plane(HPlane<T>& q, const T* __restrict__ aH, const T* __restrict__ bH,
                                             const T* __restrict__ H, const T* __restrict__ E, long long o,
                                             long long vol, long long sj) {
    q.ax = __ldg(aH + o);
    q.ay = __ldg(aH + vol + o);
    q.az = __ldg(aH + 2 * vol + o);
    q.bx = __ldg(bH + o);
    q.by = __ldg(bH + vol + o);
    q.bz = __ldg(bH + 2 * vol + o);
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
__device__ __forceinline__ void compute_E(const StencilArgs<T>& p, const EPlane<T>& cur, T& hz_im, T& hy_im,
                                          int i, int j, int k, long long o, long long vol) {
    T* __restrict__ E = p.e;
    const T cx = ((cur.hz - cur.hz_jm) - cur.hy) + cur.hy_km;
    const T cy = ((cur.hx - cur.hx_km) - cur.hz) + hz_im;
    const T cz = ((cur.hy - hy_im) - cur.hx) + cur.hx_jm;
    T ex = cur.ax * cur.ex + cur.bx * cx;
    T ey = cur.ay * cur.ey + cur.by * cy;
    T ez = cur.az * cur.ez + cur.bz * cz;
    for (int fi = 0; fi < p.nfaces; ++fi) {
        const FaceDev& f = p.f[fi];
        const int coord = (f.axis == 0) ? i : ((f.axis == 1) ? j : k);
        const int l = coord - f.lo;
        if ((unsigned)l >= (unsigned)f.n) continue;
        const long long s = slab_index_s<T>(f, l, i, j, k);
        const T* bcc = static_cast<const T*>(f.bcc);
        const T cb = bcc[l], cc = bcc[f.n + l], cck = bcc[2 * f.n + l];
        T* psi = static_cast<T*>(f.psi);
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
            ey = ey + cur.by * (cck * d1 + p1);
            ez = ez - cur.bz * (cck * d2 + p2);
        } else if (f.axis == 1) {
            ex = ex - cur.bx * (cck * d1 + p1);
            ez = ez + cur.bz * (cck * d2 + p2);
        } else {
            ex = ex + cur.bx * (cck * d1 + p1);
            ey = ey - cur.by * (cck * d2 + p2);
        }
    }
    E[o] = ex;
    E[vol + o] = ey;
    E[2 * vol + o] = ez;
    hz_im = cur.hz;
    hy_im = cur.hy;
}

template <typename T>
__global__ void __launch_bounds__(kSX* kSY) k_update_E_stream(const StencilArgs<T> p) {
    const Geom& g = p.g;
    const int k = blockIdx.x * kSX + threadIdx.x;
    const int j = blockIdx.y * kSY + threadIdx.y;
    if (k > g.nz || j > g.ny) return;
    const int i0 = blockIdx.z * p.ichunk;
    const int i1 = min(i0 + p.ichunk, g.nx + 1);
    const long long vol = g.vol, si = g.si, sj = g.sj;
    const T* __restrict__ aE = p.aE;
    const T* __restrict__ bE = p.bE;
    const T* __restrict__ E = p.e;
    const T* __restrict__ H = p.h;
    long long o = pidx(g, i0, j, k);
    T hz_im = __ldg(H + 2 * vol + o - si);
    T hy_im = __ldg(H + vol + o - si);
    EPlane<T> cur, nxt;
    load_E_plane(cur, aE, bE, E, H, o, vol, sj);
    for (int i = i0; i < i1; ++i) {
        if (i + 1 < i1) load_E_plane(nxt, aE, bE, E, H, o + si, vol, sj);
        compute_E(p, cur, hz_im, hy_im, i, j, k, o, vol);
        cur = nxt;
        o += si;
    }
}

template <typename T>
__device__ __forceinline__ void compute_H(const StencilArgs<T>& p, const HPlane<T>& cur, T& ez_ip, T& ey_ip,
                                          int i, int j, int k, long long o, long long vol) {
    T* __restrict__ H = p.h;
    const T cx = ((cur.ez_jp - cur.ez) - cur.ey_kp) + cur.ey;
    const T cy = ((cur.ex_kp - cur.ex) - ez_ip) + cur.ez;
    const T cz = ((ey_ip - cur.ey) - cur.ex_jp) + cur.ex;
    T hx = cur.ax * cur.hx - cur.bx * cx;
    T hy = cur.ay * cur.hy - cur.by * cy;
    T hz = cur.az * cur.hz - cur.bz * cz;
    for (int fi = 0; fi < p.nfaces; ++fi) {
        const FaceDev& f = p.f[fi];
        const int coord = (f.axis == 0) ? i : ((f.axis == 1) ? j : k);
        const int l = coord - f.lo;
        if ((unsigned)l >= (unsigned)f.n) continue;
        const long long s = slab_index_s<T>(f, l, i, j, k);
        const T* bcc = static_cast<const T*>(f.bcc);
        const T cb = bcc[l], cc = bcc[f.n + l], cck = bcc[2 * f.n + l];
        T* psi = static_cast<T*>(f.psi);
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
            hy = hy - cur.by * (cck * d1 + p1);
            hz = hz + cur.bz * (cck * d2 + p2);
        } else if (f.axis == 1) {
            hx = hx + cur.bx * (cck * d1 + p1);
            hz = hz - cur.bz * (cck * d2 + p2);
        } else {
            hx = hx - cur.bx * (cck * d1 + p1);
            hy = hy + cur.by * (cck * d2 + p2);
        }
    }
    H[o] = hx;
    H[vol + o] = hy;
    H[2 * vol + o] = hz;
    ez_ip = cur.ez;
    ey_ip = cur.ey;
}

template <typename T>
__global__ void __launch_bounds__(kSX* kSY) k_update_H_stream(const StencilArgs<T> p) {
    const Geom& g = p.g;
    const int k = blockIdx.x * kSX + threadIdx.x;
    const int j = blockIdx.y * kSY + threadIdx.y;
    if (k > g.nz || j > g.ny) return;
    const int i0 = blockIdx.z * p.ichunk;
    const int i1 = min(i0 + p.ichunk, g.nx + 1);
    const long long vol = g.vol, si = g.si, sj = g.sj;
    const T* __restrict__ aH = p.aH;
    const T* __restrict__ bH = p.bH;
    const T* __restrict__ H = p.h;
    const T* __restrict__ E = p.e;
    // march down: the x-neighbours (E at i+1) of the first plane
    long long o = pidx(g, i1 - 1, j, k);
    T ez_ip = __ldg(E + 2 * vol + o + si);
    T ey_ip = __ldg(E + vol + o + si);
    HPlane<T> cur, nxt;
    load_H_plane(cur, aH, bH, H, E, o, vol, sj);
    for (int i = i1 - 1; i >= i0; --i) {
        if (i - 1 >= i0) load_H_plane(nxt, aH, bH, H, E, o - si, vol, sj);
        compute_H(p, cur, ez_ip, ey_ip, i, j, k, o, vol);
        cur = nxt;
        o -= si;
    }
}

}  // namespace

template <typename T>
int stream_occupancy() {
    int a = 0, b = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_update_E_stream<T>, kSX * kSY, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_update_H_stream<T>, kSX * kSY, 0);
    const int m = a < b ? a : b;
    return m < 1 ? 1 : m;
}
template int stream_occupancy<float>();
template int stream_occupancy<double>();

StreamPlan plan_stream(const Geom& g, int sm_count, int ctas_per_sm) {
    StreamPlan s{};
    const int bx = (g.nz + 1 + kSX - 1) / kSX, by = (g.ny + 1 + kSY - 1) / kSY;
    const int nplanes = g.nx + 1;
    const int per_wave = sm_count * ctas_per_sm;
    double best = -1.0;
    int best_chunk = nplanes;
    for (int ichunk = nplanes; ichunk >= 4; --ichunk) {
        const int nch = (nplanes + ichunk - 1) / ichunk;
        const double waves = (double)bx * by * nch / per_wave;
        const double eff = waves / (double)((long long)(waves + 0.999999));
        // prefer long chunks (fewer re-loaded boundary planes) unless the
        // wave tail costs more than a few percent
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
void launch_update_E_stream(StencilArgs<T> a, const StreamPlan& sp, cudaStream_t s) {
    a.ichunk = sp.ichunk;
    k_update_E_stream<T><<<dim3(sp.grid_x, sp.grid_y, sp.grid_z), dim3(kSX, kSY, 1), 0, s>>>(a);
}

template <typename T>
void launch_update_H_stream(StencilArgs<T> a, const StreamPlan& sp, cudaStream_t s) {
    a.ichunk = sp.ichunk;
    k_update_H_stream<T><<<dim3(sp.grid_x, sp.grid_y, sp.grid_z), dim3(kSX, kSY, 1), 0, s>>>(a);
}

template void launch_update_E_stream<float>(StencilArgs<float>, const StreamPlan&, cudaStream_t);
template void launch_update_E_stream<double>(StencilArgs<double>, const StreamPlan&, cudaStream_t);
template void launch_update_H_stream<float>(StencilArgs<float>, const StreamPlan&, cudaStream_t);
template void launch_update_H_stream<double>(StencilArgs<double>, const StreamPlan&, cudaStream_t);

}  // namespace fitb
