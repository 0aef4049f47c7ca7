// Fused leapfrog step through shared-memory tiles fed by the tensor memory
// accelerator (TMA), with the CPML applied as passes over its slabs.
//
// Same arithmetic, in the same order per value, as the two-pass kernels
// (reference: numba_kernels.py:36-127 for the curl updates, cpml.py:343-516
// for the psi recursion and its correction).  Like the other fused forms the
// step reads E, H and psi from one buffer set and writes the new values to
// the other.
//
// Tile kernel.  A CTA owns a tile of TJ rows (j) by 32 cells (k) of one
// field set and marches over a chunk [i0, i1) of i planes.  One producer
// warp streams, per plane, the boxes the tile needs into a ring of NS
// shared-memory stages with 4-D tensor copies (k, j, plane, component):
//   E_old, alpha_E, beta_E  rows j0 .. j0+TJ,    cells k0 .. k0+35
//   H_old                   rows j0-1 .. j0+TJ,  cells k0-4 .. k0+35
//   alpha_H, beta_H         rows j0 .. j0+TJ-1,  cells k0 .. k0+31
// (boxes start on 16-byte boundaries; rows and cells outside the padded box
// arrive as zeros, which is what the padding holds).  TJ compute warps, for
// plane i, compute E_new(i) on the tile plus one row and one column (the
// j+1 / k+1 neighbours the H update needs; those cells are stored by the
// neighbouring tile) from stages i and i-1, keep it in a three-plane
// shared-memory ring, synchronise on a named barrier, compute H_new(i-1) of
// the tile from E_new(i-1), E_new(i) and stage i-1, then release stage i-1
// to the producer.  Every array crosses DRAM once: 96 bytes per cell in
// float32.  The first stage of a chunk (plane i0-1) carries only H; the last
// (plane i1) carries no H coefficients; E_new(i1) is computed (not stored)
// for H_new(i1-1).  A last row j = ny or column k = nz that would be a tile
// of its own is taken by the tile before it through its halo row / column.
//
// CPML.  The tile kernel has no CPML code (a few slab cells in a warp would
// otherwise run the psi recursion with most lanes idle, inside the per-plane
// barrier chain).  As in the reference's own order (fit_td.py:833-882) the
// E-side CPML follows the curl update (k_tile_cpml_E: per slab cell, every
// face of the cell in face order, psi_E update and E correction from
// H_old), then the ports write E, then every H
// cell whose update involves a slab (its own psi_H, or an E edge the E pass
// corrected) is recomputed from H_old and the final E_new with its CPML
// (k_tile_fix_boxes, the k_fix_H arithmetic over each slab extended by one
// layer on its low side).
//
// Every mbarrier wait is bounded.  When one expires the CTA records a status
// code, stops issuing copies, waits (bounded) for the copies it has in
// flight and returns; the host reads the status after the step.
#include "fused_cpml.cuh"
#include "pass_boxes.h"
#include "tile_common.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

namespace fitb {

namespace {

using tma::TK;
using tma::compute_barrier;
using tma::saddr;

struct TileMaps {
    CUtensorMap e, h, aE, bE, aH, bH;
};
static_assert(sizeof(TileMaps) == 6 * 128, "tensor map size");

// Shared-memory layout of one tile configuration.
template <typename T, int TJ, int NS>
struct TileGeo {
    static constexpr int EK = TK + 4, ER = TJ + 1;  // E, alpha_E, beta_E boxes
    static constexpr int HK = TK + 8, HR = TJ + 2;  // H box
    static constexpr int cE = ER * EK, cH = HR * HK, cC = TJ * TK;  // elements per component
    static constexpr int NK = TK + 1, NR = TJ + 1, cN = NR * NK;   // E_new ring
    static constexpr size_t al(size_t b) { return (b + 127) / 128 * 128; }
    static constexpr unsigned bytesE = 3u * cE * sizeof(T), bytesH = 3u * cH * sizeof(T),
                              bytesC = 3u * cC * sizeof(T);
    static constexpr size_t oE = 0, oH = al(bytesE), oaE = oH + al(bytesH), obE = oaE + al(bytesE),
                            oaH = obE + al(bytesE), obH = oaH + al(bytesC), stage = obH + al(bytesC);
    static constexpr size_t oN = NS * stage, oBar = oN + al(3u * 3u * cN * sizeof(T));
    static constexpr size_t smem = oBar + 2 * NS * sizeof(unsigned long long) + 4 * sizeof(int);
};

// E_new of cell (r, c) of the tile region (r <= TJ, c <= TK) at plane i.
template <typename T, int TJ, int NS>
__device__ __forceinline__ void tile_E(const Geom& g, const unsigned char* st, const unsigned char* stp, T* en, int r,
                                       int c, int i, int j, int k, bool store, T* __restrict__ Eg) {
    using G = TileGeo<T, TJ, NS>;
    const T* E = reinterpret_cast<const T*>(st + G::oE);
    const T* Hs = reinterpret_cast<const T*>(st + G::oH);
    const T* Hp = reinterpret_cast<const T*>(stp + G::oH);
    const T* aE = reinterpret_cast<const T*>(st + G::oaE);
    const T* bE = reinterpret_cast<const T*>(st + G::obE);
    const int ie = r * G::EK + c;
    const int ih = (r + 1) * G::HK + c + 4;
    const T hx = Hs[ih], hy = Hs[G::cH + ih], hz = Hs[2 * G::cH + ih];
    const T hz_jm = Hs[2 * G::cH + ih - G::HK], hx_jm = Hs[ih - G::HK];
    const T hy_km = Hs[G::cH + ih - 1], hx_km = Hs[ih - 1];
    const T hz_im = Hp[2 * G::cH + ih], hy_im = Hp[G::cH + ih];
    const T cx = ((hz - hz_jm) - hy) + hy_km;
    const T cy = ((hx - hx_km) - hz) + hz_im;
    const T cz = ((hy - hy_im) - hx) + hx_jm;
    const T ex = aE[ie] * E[ie] + bE[ie] * cx;
    const T ey = aE[G::cE + ie] * E[G::cE + ie] + bE[G::cE + ie] * cy;
    const T ez = aE[2 * G::cE + ie] * E[2 * G::cE + ie] + bE[2 * G::cE + ie] * cz;
    const int in = r * G::NK + c;
    en[in] = ex;
    en[G::cN + in] = ey;
    en[2 * G::cN + in] = ez;
    if (store) {
        const long long o = pidx(g, i, j, k), vol = g.vol;
        Eg[o] = ex;
        Eg[vol + o] = ey;
        Eg[2 * vol + o] = ez;
    }
}

// H_new of cell (r, c) at plane i from E_new(i) (enp), E_new(i+1) (enc) and
// the stage of plane i.  EDGE: a halo cell this tile owns (last row j = ny
// or last column k = nz): E_new beyond the padded edge is zero and its H
// coefficients come from global memory.
template <typename T, int TJ, int NS, bool EDGE>
__device__ __forceinline__ void tile_H(const StencilArgs<T>& p, const unsigned char* stp, const T* enp, const T* enc,
                                       int r, int c, int i, int j, int k, T* __restrict__ Hg) {
    using G = TileGeo<T, TJ, NS>;
    const T* Hs = reinterpret_cast<const T*>(stp + G::oH);
    const int in = r * G::NK + c;
    const T ex = enp[in], ey = enp[G::cN + in], ez = enp[2 * G::cN + in];
    const T ez_jp = (!EDGE || r < TJ) ? enp[2 * G::cN + in + G::NK] : T(0);
    const T ex_jp = (!EDGE || r < TJ) ? enp[in + G::NK] : T(0);
    const T ey_kp = (!EDGE || c < TK) ? enp[G::cN + in + 1] : T(0);
    const T ex_kp = (!EDGE || c < TK) ? enp[in + 1] : T(0);
    const T ey_ip = enc[G::cN + in], ez_ip = enc[2 * G::cN + in];
    const int ih = (r + 1) * G::HK + c + 4;
    const long long o = pidx(p.g, i, j, k), vol = p.g.vol;
    FCoef<T> ch;
    if constexpr (EDGE) {
        load_coef3(ch, p.aH, p.bH, o, vol);
    } else {
        const T* aH = reinterpret_cast<const T*>(stp + G::oaH);
        const T* bH = reinterpret_cast<const T*>(stp + G::obH);
        const int ic = r * TK + c;
        ch.ax = aH[ic];
        ch.ay = aH[G::cC + ic];
        ch.az = aH[2 * G::cC + ic];
        ch.bx = bH[ic];
        ch.by = bH[G::cC + ic];
        ch.bz = bH[2 * G::cC + ic];
    }
    const T cx = ((ez_jp - ez) - ey_kp) + ey;
    const T cy = ((ex_kp - ex) - ez_ip) + ez;
    const T cz = ((ey_ip - ey) - ex_jp) + ex;
    Hg[o] = ch.ax * Hs[ih] - ch.bx * cx;
    Hg[vol + o] = ch.ay * Hs[G::cH + ih] - ch.by * cy;
    Hg[2 * vol + o] = ch.az * Hs[2 * G::cH + ih] - ch.bz * cz;
}

template <typename T, int TJ, int NS, int MINB>
__global__ void __launch_bounds__(32 * (TJ + 1), sizeof(T) == 4 ? MINB : 1)
    k_step_tile(const __grid_constant__ TileMaps maps, const StencilArgs<T> p, int* status) {
    using G = TileGeo<T, TJ, NS>;
    constexpr int NC = 32 * TJ;      // compute threads
    constexpr int NX = TK + 1 + TJ;  // halo cells (row TJ, then column TK)
    static_assert(NX <= NC, "tile shape");
    extern __shared__ __align__(128) unsigned char smem[];
    const Geom& g = p.g;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int b = blockIdx.x % p.B;
    const int k0 = (blockIdx.x / p.B) * TK, j0 = blockIdx.y * TJ;
    const int i0 = blockIdx.z * p.ichunk;
    const int i1 = min(i0 + p.ichunk, g.nx + 1);
    const int nplanes = i1 - i0 + 2;  // planes i0-1 .. i1
    unsigned long long* full = reinterpret_cast<unsigned long long*>(smem + G::oBar);
    unsigned long long* empty = full + NS;
    volatile int* flags = reinterpret_cast<volatile int*>(empty + NS);  // abort, issued, first unconsumed
    T* ring = reinterpret_cast<T*>(smem + G::oN);
    if (tid == 0) {
        for (int s = 0; s < NS; ++s) {
            tma::bar_init(&full[s], 1);
            tma::bar_init(&empty[s], TJ);
        }
        flags[0] = 0;
        flags[1] = 0;
        flags[2] = nplanes;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    if (warp == TJ) {
        // producer
        if (lane == 0) {
            int t = 0;
            for (; t < nplanes; ++t) {
                if (flags[0]) break;
                const int s = t % NS;
                if (t >= NS && !tma::bar_wait(&empty[s], (unsigned)(((t / NS) + 1) & 1))) {
                    atomicExch(status, kStatusWaitTimeoutTile);
                    flags[0] = 1;
                    break;
                }
                unsigned char* st = smem + s * G::stage;
                const int plane = i0 + 1 + t;  // padded plane of i0 - 1 + t
                const bool first = t == 0, last = t == nplanes - 1;
                unsigned bytes = G::bytesH;
                if (!first) bytes += 3 * G::bytesE;
                if (!first && !last) bytes += 2 * G::bytesC;
                tma::bar_expect(&full[s], bytes);
                tma::load_4d(st + G::oH, &maps.h, k0 - 4, j0 - 1, plane, 3 * b, &full[s]);
                if (!first) {
                    tma::load_4d(st + G::oE, &maps.e, k0, j0, plane, 3 * b, &full[s]);
                    tma::load_4d(st + G::oaE, &maps.aE, k0, j0, plane, 0, &full[s]);
                    tma::load_4d(st + G::obE, &maps.bE, k0, j0, plane, 0, &full[s]);
                }
                if (!first && !last) {
                    tma::load_4d(st + G::oaH, &maps.aH, k0, j0, plane, 0, &full[s]);
                    tma::load_4d(st + G::obH, &maps.bH, k0, j0, plane, 0, &full[s]);
                }
            }
            flags[1] = t;
        }
    } else {
        // compute warps: owned cell (warp, lane), and halo cell x for the
        // first NX threads (row TJ, then column TK)
        const long long fs = 3 * g.vol * (long long)b;
        T* __restrict__ Eg = p.e_next + fs;
        T* __restrict__ Hg = p.h_next + fs;
        const int jo = j0 + warp, ko = k0 + lane;
        const bool v_own = jo <= g.ny && ko <= g.nz;
        const bool has_x = tid < NX;
        const int rx = tid <= TK ? TJ : tid - TK - 1;
        const int cx = tid <= TK ? tid : TK;
        const int jx = j0 + rx, kx = k0 + cx;
        const bool v_x = has_x && jx <= g.ny && kx <= g.nz;
        // the last row / column of the grid with no tile of its own
        const bool absorb_j = j0 + TJ == g.ny, absorb_k = k0 + TK == g.nz;
        const bool own_x = v_x && (rx == TJ ? (absorb_j && (cx < TK || absorb_k)) : absorb_k);
        for (int t = 0; t < nplanes; ++t) {
            const int s = t % NS;
            const bool ok = tma::bar_wait(&full[s], (unsigned)((t / NS) & 1));
            if (!ok) {
                atomicExch(status, kStatusWaitTimeoutTile);
                flags[0] = 1;
            }
            const int i = i0 - 1 + t;
            if (t > 0 && ok) {
                const unsigned char* st = smem + s * G::stage;
                const unsigned char* stp = smem + ((t - 1) % NS) * G::stage;
                T* en = ring + (t % 3) * 3 * G::cN;
                tile_E<T, TJ, NS>(g, st, stp, en, warp, lane, i, jo, ko, v_own && i < i1, Eg);
                if (has_x) tile_E<T, TJ, NS>(g, st, stp, en, rx, cx, i, jx, kx, own_x && i < i1, Eg);
            }
            compute_barrier(NC);
            if (flags[0]) {
                if (tid == 0) flags[2] = t;
                break;
            }
            if (t > 1) {
                const unsigned char* stp = smem + ((t - 1) % NS) * G::stage;
                const T* enp = ring + ((t - 1) % 3) * 3 * G::cN;
                const T* enc = ring + (t % 3) * 3 * G::cN;
                if (v_own) tile_H<T, TJ, NS, false>(p, stp, enp, enc, warp, lane, i - 1, jo, ko, Hg);
                if (own_x) tile_H<T, TJ, NS, true>(p, stp, enp, enc, rx, cx, i - 1, jx, kx, Hg);
            }
            if (t > 0) {
                __syncwarp();
                if (lane == 0) tma::bar_arrive(&empty[(t - 1) % NS]);
            }
        }
    }
    __syncthreads();
    // after an expired wait: the copies issued but not consumed
    if (tid == 0)
        for (int t = flags[2]; t < flags[1]; ++t) tma::bar_wait(&full[t % NS], (unsigned)((t / NS) & 1));
}

// Cell (i, j, k) of this thread and its box, or false past the box's end.
__device__ __forceinline__ bool pass_cell(const PassBoxes& bx, int& q, int& i, int& j, int& k) {
    int lo = 0, hi = bx.n - 1;  // last box with bstart <= blockIdx.x
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (bx.bstart[mid] <= (int)blockIdx.x)
            lo = mid;
        else
            hi = mid - 1;
    }
    q = lo;
    const int nk = bx.hi[q][2] - bx.lo[q][2], nj = bx.hi[q][1] - bx.lo[q][1];
    const int ncell = (bx.hi[q][0] - bx.lo[q][0]) * nj * nk;
    const int u = ((int)blockIdx.x - bx.bstart[q]) * kPassThreads + (int)threadIdx.x;
    if (u >= ncell) return false;
    const int w = u / nk;
    k = bx.lo[q][2] + (u - w * nk);
    i = bx.lo[q][0] + w / nj;
    j = bx.lo[q][1] + (w - (w / nj) * nj);
    return true;
}

// Slab index of cell (i, j, k) in face f (32-bit: slabs are far below 2^31).
__device__ __forceinline__ int slab32(const FaceDev& f, int i, int j, int k) {
    const int a = (f.axis == 0) ? i - f.lo : i;
    const int b = (f.axis == 1) ? j - f.lo : j;
    const int c = (f.axis == 2) ? k - f.lo : k;
    return (a * f.dJ + b) * f.pk + c;
}

// E-side CPML on the fused buffers (cpml.py:343-430), every face of the
// cell in face order: psi_E (components 0, 1) from the old psi and H_old,
// the corrections added to E_new.
template <typename T>
__global__ void __launch_bounds__(kPassThreads) k_tile_cpml_E(const StencilArgs<T> a, const PassBoxes bx) {
    int q, i, j, k;
    if (!pass_cell(bx, q, i, j, k)) return;
    const Geom& g = a.g;
    const int b = blockIdx.y;
    const int vol = (int)g.vol, si = (int)g.si, sj = (int)g.sj;
    const int o = (i + 2) * si + j * sj + k;
    const T* H = a.h + (long long)b * 3 * vol;
    T* E = a.e_next + (long long)b * 3 * vol;
    T ex = E[o], ey = E[vol + o], ez = E[2 * vol + o];
    const T bx_ = a.bE[o], by = a.bE[vol + o], bz = a.bE[2 * vol + o];
    unsigned mask = bx.mask[q];
    while (mask) {
        const int fq = __ffs(mask) - 1;
        mask &= mask - 1;
        const FaceDev& f = a.f[fq];
        const int l = ((f.axis == 0) ? i : ((f.axis == 1) ? j : k)) - f.lo;
        const int s = slab32(f, i, j, k);
        const T* bcc = static_cast<const T*>(f.bcc);
        const T cb = bcc[l], cc = bcc[f.n + l], cck = bcc[2 * f.n + l];
        const int sa = f.axis == 0 ? si : (f.axis == 1 ? sj : 1);
        // transverse H components of this axis: (first, second)
        const int c1 = f.axis == 2 ? vol : 2 * vol;  // Hz, Hz, Hy
        const int c2 = f.axis == 0 ? vol : 0;        // Hy, Hx, Hx
        const T d1 = H[c1 + o] - H[c1 + o - sa];
        const T d2 = H[c2 + o] - H[c2 + o - sa];
        const int slab = (int)f.slab;
        const T* psi = static_cast<const T*>(f.psi) + (long long)b * 4 * slab;
        T* psin = static_cast<T*>(f.psi_next) + (long long)b * 4 * slab;
        T p1 = psi[s] * cb;
        p1 = p1 + cc * d1;
        if (!f.air[s]) p1 = T(0);
        psin[s] = p1;
        T p2 = psi[slab + s] * cb;
        p2 = p2 + cc * d2;
        if (!f.air[slab + s]) p2 = T(0);
        psin[slab + s] = p2;
        if (f.axis == 0) {
            ey = ey + by * (cck * d1 + p1);
            ez = ez - bz * (cck * d2 + p2);
        } else if (f.axis == 1) {
            ex = ex - bx_ * (cck * d1 + p1);
            ez = ez + bz * (cck * d2 + p2);
        } else {
            ex = ex + bx_ * (cck * d1 + p1);
            ey = ey - by * (cck * d2 + p2);
        }
    }
    E[o] = ex;
    E[vol + o] = ey;
    E[2 * vol + o] = ez;
}

// H of every cell of the boxes (each slab with one more layer on its low
// side) from H_old / psi_old and the final E_new, with the cell's CPML
// faces (the k_fix_H arithmetic).
template <typename T>
__global__ void __launch_bounds__(kPassThreads) k_tile_fix_boxes(const StencilArgs<T> p, const PassBoxes bx) {
    int q, i, j, k;
    if (!pass_cell(bx, q, i, j, k)) return;
    const Geom& g = p.g;
    const int b = blockIdx.y;
    const int vol = (int)g.vol, si = (int)g.si, sj = (int)g.sj;
    const T* E = p.e_next + (long long)b * 3 * vol;
    const T* Hold = p.h + (long long)b * 3 * vol;
    T* Hn = p.h_next + (long long)b * 3 * vol;
    const int o = (i + 2) * si + j * sj + k;
    const T ex = E[o], ey = E[vol + o], ez = E[2 * vol + o];
    const T ez_jp = E[2 * vol + o + sj], ex_jp = E[o + sj];
    const T ey_kp = E[vol + o + 1], ex_kp = E[o + 1];
    const T ez_ip = E[2 * vol + o + si], ey_ip = E[vol + o + si];
    const T ax = p.aH[o], ay = p.aH[vol + o], az = p.aH[2 * vol + o];
    const T cbx = p.bH[o], cby = p.bH[vol + o], cbz = p.bH[2 * vol + o];
    const T cxh = ((ez_jp - ez) - ey_kp) + ey;
    const T cyh = ((ex_kp - ex) - ez_ip) + ez;
    const T czh = ((ey_ip - ey) - ex_jp) + ex;
    T hx = ax * Hold[o] - cbx * cxh;
    T hy = ay * Hold[vol + o] - cby * cyh;
    T hz = az * Hold[2 * vol + o] - cbz * czh;
    unsigned mask = bx.mask[q];
    while (mask) {
        const int fq = __ffs(mask) - 1;
        mask &= mask - 1;
        const FaceDev& f = p.f[fq];
        const int l = ((f.axis == 0) ? i : ((f.axis == 1) ? j : k)) - f.lo;
        const int s = slab32(f, i, j, k);
        const T* bcc = static_cast<const T*>(f.bcc);
        const T cb = bcc[l], cc = bcc[f.n + l], cck = bcc[2 * f.n + l];
        const T d1 = f.axis == 0 ? ez_ip - ez : (f.axis == 1 ? ez_jp - ez : ey_kp - ey);
        const T d2 = f.axis == 0 ? ey_ip - ey : (f.axis == 1 ? ex_jp - ex : ex_kp - ex);
        const int slab = (int)f.slab;
        const T* psi = static_cast<const T*>(f.psi) + (long long)b * 4 * slab;
        T* psin = static_cast<T*>(f.psi_next) + (long long)b * 4 * slab;
        const int s1 = 2 * slab + s, s2 = 3 * slab + s;
        T p1 = psi[s1] * cb;
        p1 = p1 + cc * d1;
        if (!f.air[s1]) p1 = T(0);
        psin[s1] = p1;
        T p2 = psi[s2] * cb;
        p2 = p2 + cc * d2;
        if (!f.air[s2]) p2 = T(0);
        psin[s2] = p2;
        if (f.axis == 0) {
            hy = hy - cby * (cck * d1 + p1);
            hz = hz + cbz * (cck * d2 + p2);
        } else if (f.axis == 1) {
            hx = hx + cbx * (cck * d1 + p1);
            hz = hz - cbz * (cck * d2 + p2);
        } else {
            hx = hx - cbx * (cck * d1 + p1);
            hy = hy + cby * (cck * d2 + p2);
        }
    }
    Hn[o] = hx;
    Hn[vol + o] = hy;
    Hn[2 * vol + o] = hz;
}

// Probe of the bounded wait: an mbarrier that nothing completes, waited on
// with `limit` tries; the expired wait sets *status and the kernel returns.
__global__ void k_wait_probe(int* status, unsigned limit) {
    __shared__ unsigned long long bar;
    if (threadIdx.x != 0) return;
    tma::bar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    for (unsigned n = 0; n < limit; ++n)
        if (tma::bar_try(&bar, 0u)) return;
    atomicExch(status, kStatusWaitTimeoutTile);
}

// Tile variants: (TJ, NS, min CTAs per SM).
template <typename T, typename F>
bool tile_dispatch(int variant, F&& f) {
    switch (variant) {
        case 0: f.template run<4, 3, 5>(); return true;
        case 1: f.template run<4, 4, 4>(); return true;
        case 2: f.template run<8, 4, 2>(); return true;
        case 3: f.template run<16, 4, 1>(); return true;
        case 4: f.template run<4, 5, 3>(); return true;
        case 5: f.template run<8, 3, 2>(); return true;
        case 6: f.template run<2, 4, 6>(); return true;
        case 7: f.template run<3, 3, 6>(); return true;
        case 8: f.template run<2, 3, 8>(); return true;
        default: return false;
    }
}

constexpr size_t kMaxSmem = 232448;  // B200 opt-in per CTA (227 KB), when the device cannot be queried

template <typename T>
struct TileInfo {
    size_t smem = 0;
    int tj = 0;
    template <int TJ, int NS, int MINB>
    void run() {
        smem = TileGeo<T, TJ, NS>::smem;
        tj = TJ;
    }
};

template <typename T>
struct TilePrepare {
    cudaError_t err = cudaSuccess;
    template <int TJ, int NS, int MINB>
    void run() {
        err = cudaFuncSetAttribute(k_step_tile<T, TJ, NS, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)TileGeo<T, TJ, NS>::smem);
    }
};

template <typename T>
struct TileOcc {
    int a = 0;
    template <int TJ, int NS, int MINB>
    void run() {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_step_tile<T, TJ, NS, MINB>, 32 * (TJ + 1),
                                                      TileGeo<T, TJ, NS>::smem);
    }
};

template <typename T>
struct TileLaunch {
    const TileMaps& m;
    const StencilArgs<T>& a;
    dim3 grid;
    int* status;
    cudaStream_t s;
    template <int TJ, int NS, int MINB>
    void run() {
        k_step_tile<T, TJ, NS, MINB><<<grid, 32 * (TJ + 1), TileGeo<T, TJ, NS>::smem, s>>>(m, a, status);
    }
};

// The CPML pass boxes of this handle's faces (pass_boxes.h).
bool pass_boxes(PassBoxes& bx, const Geom& g, const FaceDev* f, int nfaces, bool h_side) {
    PassFace pf[kMaxFaces];
    for (int q = 0; q < nfaces; ++q) pf[q] = PassFace{f[q].axis, f[q].lo, f[q].n};
    return pass_boxes(bx, g.nx, g.ny, g.nz, pf, nfaces, h_side);
}

}  // namespace

cudaError_t launch_wait_probe(int* status, unsigned limit, cudaStream_t s) {
    k_wait_probe<<<1, 32, 0, s>>>(status, limit);
    return cudaGetLastError();
}

template <typename T>
bool tile_supported(int variant) {
    TileInfo<T> f;
    if (!tile_dispatch<T>(variant, f)) return false;
    // the current device's opt-in limit per block (B200: 227 KB)
    int dev = 0, optin = 0;
    size_t limit = kMaxSmem;
    if (cudaGetDevice(&dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) == cudaSuccess && optin > 0)
        limit = (size_t)optin;
    return f.smem <= limit;
}
template bool tile_supported<float>(int);
template bool tile_supported<double>(int);

template <typename T>
cudaError_t prepare_tile(int variant) {
    TilePrepare<T> f;
    if (!tile_dispatch<T>(variant, f)) return cudaErrorInvalidValue;
    return f.err;
}
template cudaError_t prepare_tile<float>(int);
template cudaError_t prepare_tile<double>(int);

template <typename T>
int tile_occupancy(int variant) {
    TileOcc<T> f;
    tile_dispatch<T>(variant, f);
    return f.a < 1 ? 1 : f.a;
}
template int tile_occupancy<float>(int);
template int tile_occupancy<double>(int);

template <typename T>
StreamPlan plan_tile(const Geom& g, int sm_count, int ctas_per_sm, int B, int variant) {
    TileInfo<T> f;
    tile_dispatch<T>(variant, f);
    StreamPlan s{};
    s.block_y = f.tj;
    // a last column k = nz (row j = ny) that would be a tile of its own is
    // taken by the tile before it, through its halo column (row)
    s.grid_x = (g.nz % TK == 0 ? g.nz / TK : (g.nz + TK) / TK) * B;
    s.grid_y = g.ny % f.tj == 0 ? g.ny / f.tj : (g.ny + f.tj) / f.tj;
    const long long tiles = (long long)s.grid_x * s.grid_y;
    const int nplanes = g.nx + 1;
    const int per_wave = sm_count * ctas_per_sm;
    // chunks of about 16 planes measured best on 256^3 and 512^3 grids (a
    // chunk re-reads two planes; long chunks let all CTAs of a wave sweep
    // the same planes in step); among 12-20, the best wave quantisation
    double best = -1e30;
    int best_chunk = std::min(nplanes, 16);
    for (int ichunk = std::min(nplanes, 20); ichunk >= std::min(nplanes, 12); --ichunk) {
        const int nch = (nplanes + ichunk - 1) / ichunk;
        const double waves = (double)tiles * nch / per_wave;
        const double eff = waves / std::ceil(waves);
        const double score = eff - 1.0 / ichunk;
        if (score > best + 1e-9) {
            best = score;
            best_chunk = ichunk;
        }
    }
    s.ichunk = best_chunk;
    s.grid_z = (nplanes + best_chunk - 1) / best_chunk;
    return s;
}
template StreamPlan plan_tile<float>(const Geom&, int, int, int, int);
template StreamPlan plan_tile<double>(const Geom&, int, int, int, int);

template <typename T>
int launch_tile_step(StencilArgs<T> a, const StreamPlan& sp, int variant, int* status, cudaStream_t s) {
    TileInfo<T> info;
    if (!tile_dispatch<T>(variant, info)) return -1;
    const int tj = info.tj;
    TileMaps m;
    const long long nset = 3LL * a.B;
    if (!tma::encode_field_map<T>(&m.e, a.e, a.g, (int)nset, TK + 4, tj + 1) ||
        !tma::encode_field_map<T>(&m.h, a.h, a.g, (int)nset, TK + 8, tj + 2) ||
        !tma::encode_field_map<T>(&m.aE, a.aE, a.g, 3, TK + 4, tj + 1) || !tma::encode_field_map<T>(&m.bE, a.bE, a.g, 3, TK + 4, tj + 1) ||
        !tma::encode_field_map<T>(&m.aH, a.aH, a.g, 3, TK, tj) || !tma::encode_field_map<T>(&m.bH, a.bH, a.g, 3, TK, tj))
        return -2;
    a.ichunk = sp.ichunk;
    TileLaunch<T> f{m, a, dim3(sp.grid_x, sp.grid_y, sp.grid_z), status, s};
    tile_dispatch<T>(variant, f);
    return 0;
}
template int launch_tile_step<float>(StencilArgs<float>, const StreamPlan&, int, int*, cudaStream_t);
template int launch_tile_step<double>(StencilArgs<double>, const StreamPlan&, int, int*, cudaStream_t);

template <typename T>
int launch_tile_cpml_E(const StencilArgs<T>& a, cudaStream_t s) {
    if (a.nfaces == 0) return 0;
    if (3 * a.g.vol >= (1LL << 31)) return -1;  // 32-bit offsets in the passes
    PassBoxes bx;
    if (!pass_boxes(bx, a.g, a.f, a.nfaces, false)) return -1;
    if (bx.n == 0) return 0;
    k_tile_cpml_E<T><<<dim3(bx.bstart[bx.n], a.B), kPassThreads, 0, s>>>(a, bx);
    return 1;
}
template int launch_tile_cpml_E<float>(const StencilArgs<float>&, cudaStream_t);
template int launch_tile_cpml_E<double>(const StencilArgs<double>&, cudaStream_t);

template <typename T>
int launch_tile_cpml_H(const StencilArgs<T>& a, cudaStream_t s) {
    if (a.nfaces == 0) return 0;
    if (3 * a.g.vol >= (1LL << 31)) return -1;  // 32-bit offsets in the passes
    PassBoxes bx;
    if (!pass_boxes(bx, a.g, a.f, a.nfaces, true)) return -1;
    if (bx.n == 0) return 0;
    k_tile_fix_boxes<T><<<dim3(bx.bstart[bx.n], a.B), kPassThreads, 0, s>>>(a, bx);
    return 1;
}
template int launch_tile_cpml_H<float>(const StencilArgs<float>&, cudaStream_t);
template int launch_tile_cpml_H<double>(const StencilArgs<double>&, cudaStream_t);

template <typename T>
bool tile_step_fits(const StencilArgs<T>& a) {
    if (3 * a.g.vol >= (1LL << 31)) return false;  // 32-bit offsets in the CPML passes
    PassBoxes bx;
    return a.nfaces == 0 || (pass_boxes(bx, a.g, a.f, a.nfaces, false) && pass_boxes(bx, a.g, a.f, a.nfaces, true));
}
template bool tile_step_fits<float>(const StencilArgs<float>&);
template bool tile_step_fits<double>(const StencilArgs<double>&);

}  // namespace fitb
