// Leapfrog curl updates with the CFS-PML psi recursion fused in.
//
//   E^{n+1} = aE * E^n + bE * (C^T h)      then, on CPML slabs,
//             E += +-bE * (ck * dH + psi_E),  psi_E = air * (b psi_E + c dH)
//   H^{n+3/2} = aH * H - bH * (C e)        then, on CPML slabs,
//             H += +-bH * (ck * dE + psi_H),  psi_H = air * (b psi_H + c dE)
//
// Reference semantics: the fused Numba/CUDA kernels
// (src/magnelio/_operators/numba_kernels.py:36-127, :281-434) followed by
// CPMLBoundary.update_E / update_H (src/magnelio/boundaries/cpml.py:343-516).
// The in-thread curl order is the reference's: curl = +H_a - H_a' - H_b + H_b'.
//
// Thread mapping: one thread per (j, k) column of the padded box, marching
// over a chunk of i planes; k is the contiguous axis, so every warp issues
// 128-byte coalesced row segments.  Each thread updates all three
// components of its column for every field set b (coefficients are loaded
// once per cell and reused across the batch).
#include "fitb_common.cuh"

namespace fitb {

namespace {

constexpr int kBX = 32;
constexpr int kBY = 8;

template <typename T>
__device__ __forceinline__ long long slab_index(const FaceDev& f, int l, int i, int j, int k) {
    const int a = (f.axis == 0) ? l : i;
    const int b = (f.axis == 1) ? l : j;
    const int c = (f.axis == 2) ? l : k;
    return ((long long)a * f.dJ + b) * f.pk + c;
}

template <typename T>
__global__ void __launch_bounds__(kBX* kBY) k_update_E(const StencilArgs<T> p) {
    const Geom& g = p.g;
    const int k = blockIdx.x * kBX + threadIdx.x;
    const int j = blockIdx.y * kBY + threadIdx.y;
    if (k > g.nz || j > g.ny) return;
    const int i0 = blockIdx.z * p.ichunk;
    const int i1 = min(i0 + p.ichunk, g.nx + 1);
    const long long vol = g.vol;
    const long long si = g.si, sj = g.sj;
    for (int i = i0; i < i1; ++i) {
        const long long o = pidx(g, i, j, k);
        const T aex = p.aE[o], aey = p.aE[vol + o], aez = p.aE[2 * vol + o];
        const T bex = p.bE[o], bey = p.bE[vol + o], bez = p.bE[2 * vol + o];
        for (int b = 0; b < p.B; ++b) {
            T* E = p.e + (long long)b * 3 * vol;
            const T* H = p.h + (long long)b * 3 * vol;
            const T* Hx = H;
            const T* Hy = H + vol;
            const T* Hz = H + 2 * vol;
            const T hx = Hx[o], hy = Hy[o], hz = Hz[o];
            const T hz_jm = Hz[o - sj], hy_km = Hy[o - 1];
            const T hx_km = Hx[o - 1], hz_im = Hz[o - si];
            const T hy_im = Hy[o - si], hx_jm = Hx[o - sj];
            // Same accumulation order as the reference kernels.
            const T cx = ((hz - hz_jm) - hy) + hy_km;
            const T cy = ((hx - hx_km) - hz) + hz_im;
            const T cz = ((hy - hy_im) - hx) + hx_jm;
            T ex = aex * E[o] + bex * cx;
            T ey = aey * E[vol + o] + bey * cy;
            T ez = aez * E[2 * vol + o] + bez * cz;
            for (int fi = 0; fi < p.nfaces; ++fi) {
                const FaceDev& f = p.f[fi];
                const int coord = (f.axis == 0) ? i : ((f.axis == 1) ? j : k);
                const int l = coord - f.lo;
                if ((unsigned)l >= (unsigned)f.n) continue;
                const long long s = slab_index<T>(f, l, i, j, k);
                const T* bcc = static_cast<const T*>(f.bcc);
                const T cb = bcc[l], cc = bcc[f.n + l], cck = bcc[2 * f.n + l];
                T* psi = static_cast<T*>(f.psi) + (long long)b * 4 * f.slab;
                T d1, d2;
                if (f.axis == 0) {
                    d1 = hz - hz_im;  // psi_Ey, Ey +=
                    d2 = hy - hy_im;  // psi_Ez, Ez -=
                } else if (f.axis == 1) {
                    d1 = hz - hz_jm;  // psi_Ex, Ex -=
                    d2 = hx - hx_jm;  // psi_Ez, Ez +=
                } else {
                    d1 = hy - hy_km;  // psi_Ex, Ex +=
                    d2 = hx - hx_km;  // psi_Ey, Ey -=
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
                    ey = ey + bey * (cck * d1 + p1);
                    ez = ez - bez * (cck * d2 + p2);
                } else if (f.axis == 1) {
                    ex = ex - bex * (cck * d1 + p1);
                    ez = ez + bez * (cck * d2 + p2);
                } else {
                    ex = ex + bex * (cck * d1 + p1);
                    ey = ey - bey * (cck * d2 + p2);
                }
            }
            E[o] = ex;
            E[vol + o] = ey;
            E[2 * vol + o] = ez;
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kBX* kBY) k_update_H(const StencilArgs<T> p) {
    const Geom& g = p.g;
    const int k = blockIdx.x * kBX + threadIdx.x;
    const int j = blockIdx.y * kBY + threadIdx.y;
    if (k > g.nz || j > g.ny) return;
    const int i0 = blockIdx.z * p.ichunk;
    const int i1 = min(i0 + p.ichunk, g.nx + 1);
    const long long vol = g.vol;
    const long long si = g.si, sj = g.sj;
    for (int i = i0; i < i1; ++i) {
        const long long o = pidx(g, i, j, k);
        const T ahx = p.aH[o], ahy = p.aH[vol + o], ahz = p.aH[2 * vol + o];
        const T bhx = p.bH[o], bhy = p.bH[vol + o], bhz = p.bH[2 * vol + o];
        for (int b = 0; b < p.B; ++b) {
            const T* E = p.e + (long long)b * 3 * vol;
            T* H = p.h + (long long)b * 3 * vol;
            const T* Ex = E;
            const T* Ey = E + vol;
            const T* Ez = E + 2 * vol;
            const T ex = Ex[o], ey = Ey[o], ez = Ez[o];
            const T ez_jp = Ez[o + sj], ey_kp = Ey[o + 1];
            const T ex_kp = Ex[o + 1], ez_ip = Ez[o + si];
            const T ey_ip = Ey[o + si], ex_jp = Ex[o + sj];
            const T cx = ((ez_jp - ez) - ey_kp) + ey;
            const T cy = ((ex_kp - ex) - ez_ip) + ez;
            const T cz = ((ey_ip - ey) - ex_jp) + ex;
            T hx = ahx * H[o] - bhx * cx;
            T hy = ahy * H[vol + o] - bhy * cy;
            T hz = ahz * H[2 * vol + o] - bhz * cz;
            for (int fi = 0; fi < p.nfaces; ++fi) {
                const FaceDev& f = p.f[fi];
                const int coord = (f.axis == 0) ? i : ((f.axis == 1) ? j : k);
                const int l = coord - f.lo;
                if ((unsigned)l >= (unsigned)f.n) continue;
                const long long s = slab_index<T>(f, l, i, j, k);
                const T* bcc = static_cast<const T*>(f.bcc);
                const T cb = bcc[l], cc = bcc[f.n + l], cck = bcc[2 * f.n + l];
                T* psi = static_cast<T*>(f.psi) + (long long)b * 4 * f.slab;
                T d1, d2;
                if (f.axis == 0) {
                    d1 = ez_ip - ez;  // psi_Hy, Hy -=
                    d2 = ey_ip - ey;  // psi_Hz, Hz +=
                } else if (f.axis == 1) {
                    d1 = ez_jp - ez;  // psi_Hx, Hx +=
                    d2 = ex_jp - ex;  // psi_Hz, Hz -=
                } else {
                    d1 = ey_kp - ey;  // psi_Hx, Hx -=
                    d2 = ex_kp - ex;  // psi_Hy, Hy +=
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
                    hy = hy - bhy * (cck * d1 + p1);
                    hz = hz + bhz * (cck * d2 + p2);
                } else if (f.axis == 1) {
                    hx = hx + bhx * (cck * d1 + p1);
                    hz = hz - bhz * (cck * d2 + p2);
                } else {
                    hx = hx - bhx * (cck * d1 + p1);
                    hy = hy + bhy * (cck * d2 + p2);
                }
            }
            H[o] = hx;
            H[vol + o] = hy;
            H[2 * vol + o] = hz;
        }
    }
}

template <typename T>
__global__ void k_pack(const T* __restrict__ flat, T* __restrict__ padded, Geom g, int comp) {
    int ni, nj, nk;
    comp_shape(g, comp, ni, nj, nk);
    const long long n = (long long)ni * nj * nk;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(t % nk);
        const long long r = t / nk;
        const int j = (int)(r % nj);
        const int i = (int)(r / nj);
        padded[pidx(g, i, j, k)] = flat[t];
    }
}

template <typename T>
__global__ void k_unpack(const T* __restrict__ padded, T* __restrict__ flat, Geom g, int comp) {
    int ni, nj, nk;
    comp_shape(g, comp, ni, nj, nk);
    const long long n = (long long)ni * nj * nk;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(t % nk);
        const long long r = t / nk;
        const int j = (int)(r % nj);
        const int i = (int)(r / nj);
        flat[t] = padded[pidx(g, i, j, k)];
    }
}

__global__ void k_advance(long long* step) { step[0] += 1; }

template <typename T>
__global__ void k_energy_partial(const T* __restrict__ e, const T* __restrict__ h,
                                 const T* __restrict__ meps, const T* __restrict__ mmu,
                                 long long n3, double* __restrict__ partials) {
    double acc = 0.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n3;
         t += (long long)gridDim.x * blockDim.x) {
        const double ev = (double)e[t], hv = (double)h[t];
        acc += (double)meps[t] * ev * ev + (double)mmu[t] * hv * hv;
    }
    __shared__ double red[256];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) partials[blockIdx.x] = red[0];
}

__global__ void k_energy_final(const double* __restrict__ partials, int n, double* out) {
    __shared__ double red[256];
    double acc = 0.0;
    for (int t = threadIdx.x; t < n; t += blockDim.x) acc += partials[t];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = 0.5 * red[0];
}

}  // namespace

template <typename T>
void launch_update_E(const StencilArgs<T>& a, cudaStream_t s) {
    dim3 block(kBX, kBY, 1);
    dim3 grid((a.g.nz + 1 + kBX - 1) / kBX, (a.g.ny + 1 + kBY - 1) / kBY,
              (a.g.nx + 1 + a.ichunk - 1) / a.ichunk);
    k_update_E<T><<<grid, block, 0, s>>>(a);
}

template <typename T>
void launch_update_H(const StencilArgs<T>& a, cudaStream_t s) {
    dim3 block(kBX, kBY, 1);
    dim3 grid((a.g.nz + 1 + kBX - 1) / kBX, (a.g.ny + 1 + kBY - 1) / kBY,
              (a.g.nx + 1 + a.ichunk - 1) / a.ichunk);
    k_update_H<T><<<grid, block, 0, s>>>(a);
}

template <typename T>
void launch_pack(const T* flat, T* padded, const Geom& g, int comp, long long flat_off,
                 cudaStream_t s) {
    k_pack<T><<<1184, 256, 0, s>>>(flat + flat_off, padded, g, comp);
}

template <typename T>
void launch_unpack(const T* padded, T* flat, const Geom& g, int comp, long long flat_off,
                   cudaStream_t s) {
    k_unpack<T><<<1184, 256, 0, s>>>(padded, flat + flat_off, g, comp);
}

void launch_advance(long long* step, cudaStream_t s) { k_advance<<<1, 1, 0, s>>>(step); }

template <typename T>
void launch_energy(const T* e, const T* h, const T* meps, const T* mmu, const Geom& g, int b,
                   long long e_block, double* partials, int nblocks, double* out,
                   cudaStream_t s) {
    const T* eb = e + (long long)b * e_block;
    const T* hb = h + (long long)b * e_block;
    k_energy_partial<T><<<nblocks, 256, 0, s>>>(eb, hb, meps, mmu, e_block, partials);
    k_energy_final<<<1, 256, 0, s>>>(partials, nblocks, out);
}

#define FITB_INST(T)                                                                           \
    template void launch_update_E<T>(const StencilArgs<T>&, cudaStream_t);                    \
    template void launch_update_H<T>(const StencilArgs<T>&, cudaStream_t);                    \
    template void launch_pack<T>(const T*, T*, const Geom&, int, long long, cudaStream_t);     \
    template void launch_unpack<T>(const T*, T*, const Geom&, int, long long, cudaStream_t);   \
    template void launch_energy<T>(const T*, const T*, const T*, const T*, const Geom&, int,    \
                                   long long, double*, int, double*, cudaStream_t);
FITB_INST(float)
FITB_INST(double)
#undef FITB_INST

}  // namespace fitb
