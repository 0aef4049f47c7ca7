// Fused leapfrog step through TMA-fed shared-memory tiles with the CPML
// inside the march: the slab step.
//
// Same arithmetic, in the same order per value, as the two-pass kernels
// (reference: numba_kernels.py:36-127 for the curl updates, cpml.py:343-516
// for the psi recursion and its correction, faces in boundary order).  The
// step reads E, H and psi from one buffer set and writes the new values to
// the other, like the other fused forms.
//
// Work units.  A unit is a tile of TJ rows (j) by 32 cells (k) of one field
// set over a chunk [i0, i1) of i planes, marched as in the tile step
// (stencil_tile.cu): a producer warp streams each plane's boxes into a ring
// of NS shared-memory stages with 4-D tensor copies, TJ compute warps
// compute E_new of the tile plus its j+1 row and k+1 column, keep three
// planes of E_new in shared memory and compute H_new one plane behind.
// The host lists the units by the number of CPML faces their cells touch
// (0, 1, 2, 3, or up to 6 on grids small enough for both faces of an axis
// to reach one unit) and each list runs as one launch of the kernel built
// for that many face slots, so the units without CPML run the plain march
// at its full occupancy.
//
// Face slots.  For every face slot the producer adds, per plane, the
// unit's boxes of that face's padded psi slab (rows of pk entries, 16-byte
// aligned): psi_E on the E box rows (j0 .. j0+TJ) and psi_H on the tile
// rows, plus the matching air-mask boxes (bytes) when any face carries PEC
// masks; an x face only on the planes inside its slab.  The compute warps
// correct E_new of every cell inside a slot's slab before it enters the
// E_new ring (so the H update reads corrected E, as in the reference's
// order: curl update, CPML correction, then H), correct H_new after its
// curl update, and write psi_next of the cells they own.  Corrections run
// in slot order, which is the boundary order of the faces.
//
// Every mbarrier wait is bounded.  When one expires the CTA records a status
// code, stops issuing copies, waits (bounded) for the copies it has in
// flight and returns; the host reads the status after the step.
#include "fused_cpml.cuh"
#include "tile_common.cuh"

#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <vector>

namespace fitb {

namespace {

using tma::TK;
constexpr int kSlotMax = 6;  // two faces per axis
constexpr int PW = 36;  // psi box row (entries): 33 cells + up to 3 of alignment offset
constexpr int AW = 48;  // air box row (bytes): 33 cells + up to 15 of alignment offset
constexpr size_t kSmemPerSM = 233472;  // B200: 228 KB of shared memory per SM
constexpr size_t kSmemPerCTA = 1024;   // reserved per resident CTA

struct SlabMaps {
    CUtensorMap e, h, aE, bE, aH, bH;
    CUtensorMap psiE[kMaxFaces], psiH[kMaxFaces], airE[kMaxFaces], airH[kMaxFaces];
};

// One face slot of a unit, resolved once per CTA.
template <typename T>
struct Slot {
    int axis, lo, n, pk, dJ, face;
    int c0, c1;  // psi box x / row start coordinates
    int ca0;     // air box x start
    int co, ca;  // box column of cell column 0 (psi, air)
    long long slab;
    const T* bcc;
    const T* psi;   // this field set's psi (old), [4][slab]
    T* psin;        // this field set's psi_next
    const unsigned char* air;  // [4][slab]
};

template <typename T, int TJ, int NS, int NSLOT, bool AIR, int CK, int NB>
struct SlabGeo {
    static constexpr int EK = TK + 4, ER = TJ + 1;  // E, alpha_E, beta_E boxes
    static constexpr int HK = TK + 8, HR = TJ + 2;  // H box
    static constexpr int cE = ER * EK, cH = HR * HK, cC = TJ * TK;
    static constexpr int NK = TK + 1, NR = TJ + 1, cN = NR * NK;  // E_new ring
    static constexpr int cPE = ER * PW, cPH = TJ * PW, cAE = ER * AW, cAH = TJ * AW;  // per component
    // coefficient boxes: the field dtype, or 16-bit (CK != kCoefNative) with
    // E rows of 40 entries (a 16-byte multiple covering the 33 cells)
    static constexpr int CB = CK == kCoefNative ? (int)sizeof(T) : 2;
    static constexpr int EKc = CK == kCoefNative ? EK : 40, cCE = ER * EKc;
    static constexpr size_t al(size_t b) { return (b + 127) / 128 * 128; }
    // E and H boxes of the NB field sets one after the other (one copy of
    // 3 NB components each), psi boxes one copy per field set; the
    // coefficient and air-mask boxes once for all of them.  Every tensor
    // copy lands on a 128-byte boundary: the per-set psi boxes at a stride
    // of setPE / setPH rounded up to 128 bytes.
    static constexpr unsigned setE = 3u * cE * sizeof(T), setH = 3u * cH * sizeof(T);
    static constexpr unsigned setPE = (unsigned)al(2u * cPE * sizeof(T)), setPH = (unsigned)al(2u * cPH * sizeof(T));
    static constexpr unsigned bytesE = NB * setE, bytesH = NB * setH, bytesCE = 3u * cCE * CB, bytesC = 3u * cC * CB;
    // bytes the copies deliver (the expected transaction counts)
    static constexpr unsigned bytesPE = NB * 2u * cPE * sizeof(T), bytesPH = NB * 2u * cPH * sizeof(T),
                              bytesAE = 2u * cAE, bytesAH = 2u * cAH;
    static constexpr size_t oE = 0, oH = al(bytesE), oaE = oH + al(bytesH), obE = oaE + al(bytesCE),
                            oaH = obE + al(bytesCE), obH = oaH + al(bytesC), oS = obH + al(bytesC);
    // within a slot: psi_E, psi_H, air_E, air_H
    static constexpr size_t sPE = 0, sPH = NB * setPE, sAE = sPH + NB * setPH,
                            sAH = sAE + (AIR ? al(bytesAE) : 0), slot = sAH + (AIR ? al(bytesAH) : 0);
    static_assert(oH % 128 == 0 && oaE % 128 == 0 && obE % 128 == 0 && oaH % 128 == 0 && obH % 128 == 0 &&
                      oS % 128 == 0 && setPE % 128 == 0 && setPH % 128 == 0 && sAE % 128 == 0 &&
                      sAH % 128 == 0 && slot % 128 == 0,
                  "tensor copy destinations on 128-byte boundaries");
    static constexpr size_t stage = oS + NSLOT * slot;
    // E_new ring: 3 planes x NB field sets x 3 components
    static constexpr size_t oN = NS * stage, oSl = oN + al(3u * NB * 3u * cN * sizeof(T));
    static constexpr size_t oBar = oSl + al((NSLOT > 0 ? NSLOT : 1) * sizeof(Slot<T>));
    static constexpr size_t smem = oBar + 2 * NS * sizeof(unsigned long long) + 4 * sizeof(int);
    // resident CTAs per SM that the shared memory allows (launch bound)
    static constexpr int minb() {
        const size_t c = kSmemPerSM / (smem + kSmemPerCTA);
        return c < 1 ? 1 : (c > 8 ? 8 : (int)c);
    }
};

// CPML of E_new of cell (r, c) of the tile region at plane i (cpml.py:343-430).
template <typename T, int TJ, int NS, int NSLOT, bool AIR, int CK, int NB>
__device__ __forceinline__ void slab_E(const Slot<T>* sl, const unsigned char* st, int sb, int r, int c, int i, int j,
                                       int k,
                                       T hx, T hy, T hz, T hz_jm, T hx_jm, T hy_km, T hx_km, T hz_im, T hy_im, T bx,
                                       T by, T bz, T& ex, T& ey, T& ez, bool store) {
    using G = SlabGeo<T, TJ, NS, NSLOT, AIR, CK, NB>;
#pragma unroll
    for (int s = 0; s < NSLOT; ++s) {
        const Slot<T>& f = sl[s];
        const int a = f.axis;
        const int l = (a == 0 ? i : (a == 1 ? j : k)) - f.lo;
        if ((unsigned)l >= (unsigned)f.n) continue;
        const unsigned char* ss = st + G::oS + s * G::slot;
        const T* ps = reinterpret_cast<const T*>(ss + G::sPE + sb * G::setPE);
        const int q = r * PW + c + f.co;
        const T cb = __ldg(f.bcc + l), cc = __ldg(f.bcc + f.n + l), cck = __ldg(f.bcc + 2 * f.n + l);
        const T d1 = a == 0 ? hz - hz_im : (a == 1 ? hz - hz_jm : hy - hy_km);
        const T d2 = a == 0 ? hy - hy_im : (a == 1 ? hx - hx_jm : hx - hx_km);
        T p1 = ps[q] * cb;
        p1 = p1 + cc * d1;
        T p2 = ps[G::cPE + q] * cb;
        p2 = p2 + cc * d2;
        if constexpr (AIR) {
            const unsigned char* am = ss + G::sAE;
            const int qa = r * AW + c + f.ca;
            if (!am[qa]) p1 = T(0);
            if (!am[G::cAE + qa]) p2 = T(0);
        }
        if (store) {
            const long long o =
                ((long long)(a == 0 ? l : i) * f.dJ + (a == 1 ? l : j)) * f.pk + (a == 2 ? l : k);
            T* pn = f.psin + sb * 4 * f.slab;
            pn[o] = p1;
            pn[f.slab + o] = p2;
        }
        if (a == 0) {
            ey = ey + by * (cck * d1 + p1);
            ez = ez - bz * (cck * d2 + p2);
        } else if (a == 1) {
            ex = ex - bx * (cck * d1 + p1);
            ez = ez + bz * (cck * d2 + p2);
        } else {
            ex = ex + bx * (cck * d1 + p1);
            ey = ey - by * (cck * d2 + p2);
        }
    }
}

// CPML of H_new of cell (r, c) at plane i (cpml.py:432-516), psi components
// 2 and 3.  EDGE: a cell outside the staged tile rows / columns (the last
// row j = ny or column k = nz absorbed by this tile); its psi and air come
// from global memory.
template <typename T, int TJ, int NS, int NSLOT, bool AIR, int CK, int NB, bool EDGE>
__device__ __forceinline__ void slab_H(const Slot<T>* sl, const unsigned char* stp, int sb, int r, int c, int i, int j,
                                       int k,
                                       T ex, T ey, T ez, T ez_jp, T ex_jp, T ey_kp, T ex_kp, T ez_ip, T ey_ip, T bx,
                                       T by, T bz, T& hx, T& hy, T& hz) {
    using G = SlabGeo<T, TJ, NS, NSLOT, AIR, CK, NB>;
#pragma unroll
    for (int s = 0; s < NSLOT; ++s) {
        const Slot<T>& f = sl[s];
        const int a = f.axis;
        const int l = (a == 0 ? i : (a == 1 ? j : k)) - f.lo;
        if ((unsigned)l >= (unsigned)f.n) continue;
        const T cb = __ldg(f.bcc + l), cc = __ldg(f.bcc + f.n + l), cck = __ldg(f.bcc + 2 * f.n + l);
        const T d1 = a == 0 ? ez_ip - ez : (a == 1 ? ez_jp - ez : ey_kp - ey);
        const T d2 = a == 0 ? ey_ip - ey : (a == 1 ? ex_jp - ex : ex_kp - ex);
        const long long o = ((long long)(a == 0 ? l : i) * f.dJ + (a == 1 ? l : j)) * f.pk + (a == 2 ? l : k);
        T s1, s2;
        bool air1 = true, air2 = true;
        if constexpr (EDGE) {
            const T* po = f.psi + sb * 4 * f.slab;
            s1 = po[2 * f.slab + o];
            s2 = po[3 * f.slab + o];
            if constexpr (AIR) {
                air1 = f.air[2 * f.slab + o] != 0;
                air2 = f.air[3 * f.slab + o] != 0;
            }
        } else {
            const unsigned char* ss = stp + G::oS + s * G::slot;
            const T* ps = reinterpret_cast<const T*>(ss + G::sPH + sb * G::setPH);
            const int q = r * PW + c + f.co;
            s1 = ps[q];
            s2 = ps[G::cPH + q];
            if constexpr (AIR) {
                const unsigned char* am = ss + G::sAH;
                const int qa = r * AW + c + f.ca;
                air1 = am[qa] != 0;
                air2 = am[G::cAH + qa] != 0;
            }
        }
        T p1 = s1 * cb;
        p1 = p1 + cc * d1;
        if (!air1) p1 = T(0);
        T p2 = s2 * cb;
        p2 = p2 + cc * d2;
        if (!air2) p2 = T(0);
        T* pn = f.psin + sb * 4 * f.slab;
        pn[2 * f.slab + o] = p1;
        pn[3 * f.slab + o] = p2;
        if (a == 0) {
            hy = hy - by * (cck * d1 + p1);
            hz = hz + bz * (cck * d2 + p2);
        } else if (a == 1) {
            hx = hx + bx * (cck * d1 + p1);
            hz = hz - bz * (cck * d2 + p2);
        } else {
            hx = hx - bx * (cck * d1 + p1);
            hy = hy + by * (cck * d2 + p2);
        }
    }
}

// Three components (stride `stride` entries) of one staged coefficient box
// at entry q: the field dtype, or 16-bit storage times the per-component
// power-of-two scale cs[0..2] (the compact storage of fitb_set_coeff_storage,
// decoded as the stream kernels decode it).
template <typename T, int CK>
__device__ __forceinline__ void coef3(const unsigned char* box, int stride, int q, const float* cs, T& x, T& y,
                                      T& z) {
    if constexpr (CK == kCoefNative) {
        const T* a = reinterpret_cast<const T*>(box);
        x = a[q];
        y = a[stride + q];
        z = a[2 * stride + q];
    } else {
        const unsigned short* a = reinterpret_cast<const unsigned short*>(box);
        x = (T)__half2float(__ushort_as_half(a[q])) * (T)cs[0];
        y = (T)__half2float(__ushort_as_half(a[stride + q])) * (T)cs[1];
        z = (T)__half2float(__ushort_as_half(a[2 * stride + q])) * (T)cs[2];
    }
}

// E_new of cell (r, c) of the tile region (r <= TJ, c <= TK) at plane i,
// CPML-corrected; stored to global memory (with psi_next) when `store`.
template <typename T, int TJ, int NS, int NSLOT, bool AIR, int CK, int NB>
__device__ __forceinline__ void step_E(const StencilArgs<T>& p, const Slot<T>* sl, const unsigned char* st,
                                       const unsigned char* stp, int sb, T* en, int r, int c, int i, int j, int k,
                                       bool store, T* __restrict__ Eg) {
    using G = SlabGeo<T, TJ, NS, NSLOT, AIR, CK, NB>;
    const Geom& g = p.g;
    const T* E = reinterpret_cast<const T*>(st + G::oE + sb * G::setE);
    const T* Hs = reinterpret_cast<const T*>(st + G::oH + sb * G::setH);
    const T* Hp = reinterpret_cast<const T*>(stp + G::oH + sb * G::setH);
    const int ie = r * G::EK + c;
    const int ic = r * G::EKc + c;
    const int ih = (r + 1) * G::HK + c + 4;
    const T hx = Hs[ih], hy = Hs[G::cH + ih], hz = Hs[2 * G::cH + ih];
    const T hz_jm = Hs[2 * G::cH + ih - G::HK], hx_jm = Hs[ih - G::HK];
    const T hy_km = Hs[G::cH + ih - 1], hx_km = Hs[ih - 1];
    const T hz_im = Hp[2 * G::cH + ih], hy_im = Hp[G::cH + ih];
    const T cx = ((hz - hz_jm) - hy) + hy_km;
    const T cy = ((hx - hx_km) - hz) + hz_im;
    const T cz = ((hy - hy_im) - hx) + hx_jm;
    T ax, ay, az, bx, by, bz;
    coef3<T, CK>(st + G::oaE, G::cCE, ic, p.cs + 0, ax, ay, az);
    coef3<T, CK>(st + G::obE, G::cCE, ic, p.cs + 4, bx, by, bz);
    T ex = ax * E[ie] + bx * cx;
    T ey = ay * E[G::cE + ie] + by * cy;
    T ez = az * E[2 * G::cE + ie] + bz * cz;
    if constexpr (NSLOT > 0)
        slab_E<T, TJ, NS, NSLOT, AIR, CK, NB>(sl, st, sb, r, c, i, j, k, hx, hy, hz, hz_jm, hx_jm, hy_km, hx_km, hz_im,
                                              hy_im, bx, by, bz, ex, ey, ez, store);
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
// the stage of plane i, CPML-corrected.  EDGE: a halo cell this tile owns
// (last row j = ny or last column k = nz): E_new beyond the padded edge is
// zero and its coefficients, psi and air come from global memory.
template <typename T, int TJ, int NS, int NSLOT, bool AIR, int CK, int NB, bool EDGE>
__device__ __forceinline__ void step_H(const StencilArgs<T>& p, const Slot<T>* sl, const unsigned char* stp, int sb,
                                       const T* enp, const T* enc, int r, int c, int i, int j, int k,
                                       T* __restrict__ Hg) {
    using G = SlabGeo<T, TJ, NS, NSLOT, AIR, CK, NB>;
    const T* Hs = reinterpret_cast<const T*>(stp + G::oH + sb * G::setH);
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
        if constexpr (CK == kCoefNative) {
            load_coef3(ch, p.aH, p.bH, o, vol);
        } else {
            const unsigned short *qa = p.cq[2], *qb = p.cq[3];
            ch.ax = (T)__half2float(__ushort_as_half(qa[o])) * (T)p.cs[8];
            ch.ay = (T)__half2float(__ushort_as_half(qa[vol + o])) * (T)p.cs[9];
            ch.az = (T)__half2float(__ushort_as_half(qa[2 * vol + o])) * (T)p.cs[10];
            ch.bx = (T)__half2float(__ushort_as_half(qb[o])) * (T)p.cs[12];
            ch.by = (T)__half2float(__ushort_as_half(qb[vol + o])) * (T)p.cs[13];
            ch.bz = (T)__half2float(__ushort_as_half(qb[2 * vol + o])) * (T)p.cs[14];
        }
    } else {
        const int ic = r * TK + c;
        coef3<T, CK>(stp + G::oaH, G::cC, ic, p.cs + 8, ch.ax, ch.ay, ch.az);
        coef3<T, CK>(stp + G::obH, G::cC, ic, p.cs + 12, ch.bx, ch.by, ch.bz);
    }
    const T cx = ((ez_jp - ez) - ey_kp) + ey;
    const T cy = ((ex_kp - ex) - ez_ip) + ez;
    const T cz = ((ey_ip - ey) - ex_jp) + ex;
    T hx = ch.ax * Hs[ih] - ch.bx * cx;
    T hy = ch.ay * Hs[G::cH + ih] - ch.by * cy;
    T hz = ch.az * Hs[2 * G::cH + ih] - ch.bz * cz;
    if constexpr (NSLOT > 0)
        slab_H<T, TJ, NS, NSLOT, AIR, CK, NB, EDGE>(sl, stp, sb, r, c, i, j, k, ex, ey, ez, ez_jp, ex_jp, ey_kp, ex_kp,
                                                    ez_ip, ey_ip, ch.bx, ch.by, ch.bz, hx, hy, hz);
    Hg[o] = hx;
    Hg[vol + o] = hy;
    Hg[2 * vol + o] = hz;
}

// Units: x = k tile, y = j tile, z = i chunk, w = the face of slot s in bits
// 4s .. 4s+3.  A CTA marches NB field sets b0 .. b0+NB-1 of its unit through
// the same coefficient boxes, with TJ compute warps per field set;
// blockIdx.x = unit * (B / NB) + b0 / NB.
template <typename T, int TJ, int NS, int NSLOT, bool AIR, int CK, int NB>
__global__ void __launch_bounds__(32 * (TJ * NB + 1), SlabGeo<T, TJ, NS, NSLOT, AIR, CK, NB>::minb())
    k_step_slab(const __grid_constant__ SlabMaps maps, const StencilArgs<T> p, const int4* __restrict__ units,
                int* status) {
    using G = SlabGeo<T, TJ, NS, NSLOT, AIR, CK, NB>;
    constexpr int NC = 32 * TJ * NB;  // compute threads
    constexpr int NX = TK + 1 + TJ;   // halo cells of a field set (row TJ, then column TK)
    static_assert(NX <= 32 * TJ, "tile shape");
    extern __shared__ __align__(128) unsigned char smem[];
    const Geom& g = p.g;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int ng = p.B / NB;  // field-set groups
    const int b = (blockIdx.x % ng) * NB;  // first field set of the CTA
    const int4 u = units[blockIdx.x / ng];
    const int k0 = (u.x & 0xffff) * TK, j0 = (u.x >> 16) * TJ;
    const int i0 = u.y, i1 = u.z;
    const int nplanes = i1 - i0 + 2;  // planes i0-1 .. i1
    unsigned long long* full = reinterpret_cast<unsigned long long*>(smem + G::oBar);
    unsigned long long* empty = full + NS;
    volatile int* flags = reinterpret_cast<volatile int*>(empty + NS);  // abort, issued, first unconsumed
    T* ring = reinterpret_cast<T*>(smem + G::oN);
    Slot<T>* sl = reinterpret_cast<Slot<T>*>(smem + G::oSl);
    if (tid < NSLOT) {
        const int fq = (u.w >> (4 * tid)) & 15;
        const FaceDev& f = p.f[fq < kMaxFaces ? fq : 0];
        Slot<T> s;
        s.face = fq;
        s.axis = f.axis;
        s.lo = f.lo;
        s.n = f.n;
        s.pk = f.pk;
        s.dJ = f.dJ;
        s.slab = f.slab;
        s.c0 = k0;
        s.c1 = j0;
        s.ca0 = k0;
        s.co = 0;
        s.ca = 0;
        if (f.axis == 1) s.c1 = j0 - f.lo;
        if (f.axis == 2) {
            const int d = k0 - f.lo;  // box column of cell column 0, before alignment
            s.c0 = d & ~3;            // 16-byte aligned start (floor, also for d < 0)
            s.ca0 = d & ~15;
            s.co = d - s.c0;
            s.ca = d - s.ca0;
        }
        s.bcc = static_cast<const T*>(f.bcc);
        s.psi = static_cast<const T*>(f.psi) + (long long)b * 4 * f.slab;  // field set b; b+q at + 4 q slab
        s.psin = static_cast<T*>(f.psi_next) + (long long)b * 4 * f.slab;
        s.air = f.air;
        if (fq >= kMaxFaces) s.n = 0;  // an empty slot of a larger-capacity launch: never active
        sl[tid] = s;
    }
    if (tid == 0) {
        for (int s = 0; s < NS; ++s) {
            tma::bar_init(&full[s], 1);
            tma::bar_init(&empty[s], TJ * NB);
        }
        flags[0] = 0;
        flags[1] = 0;
        flags[2] = nplanes;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    if (warp == TJ * NB) {
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
                const int plane = i0 + 1 + t;  // padded plane of cell plane ip = i0 - 1 + t
                const int ip = i0 - 1 + t;
                const bool first = t == 0, last = t == nplanes - 1;
                unsigned bytes = G::bytesH;
                if (!first) bytes += G::bytesE + 2 * G::bytesCE;
                if (!first && !last) bytes += 2 * G::bytesC;
                unsigned smask = 0;  // slots with boxes on this plane
#pragma unroll
                for (int q = 0; q < NSLOT; ++q) {
                    const Slot<T>& f = sl[q];
                    if (!first && f.n > 0 && (f.axis != 0 || (unsigned)(ip - f.lo) < (unsigned)f.n)) {
                        smask |= 1u << q;
                        bytes += G::bytesPE + (AIR ? G::bytesAE : 0u);
                        if (!last) bytes += G::bytesPH + (AIR ? G::bytesAH : 0u);
                    }
                }
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
#pragma unroll
                for (int q = 0; q < NSLOT; ++q) {
                    if (!(smask >> q & 1)) continue;
                    const Slot<T>& f = sl[q];
                    const int pl = f.axis == 0 ? ip - f.lo : ip;
                    unsigned char* ss = st + G::oS + q * G::slot;
#pragma unroll
                    for (int m = 0; m < NB; ++m)
                        tma::load_4d(ss + G::sPE + m * G::setPE, &maps.psiE[f.face], f.c0, f.c1, pl, 4 * (b + m),
                                     &full[s]);
                    if constexpr (AIR) tma::load_4d(ss + G::sAE, &maps.airE[f.face], f.ca0, f.c1, pl, 0, &full[s]);
                    if (!last) {
#pragma unroll
                        for (int m = 0; m < NB; ++m)
                            tma::load_4d(ss + G::sPH + m * G::setPH, &maps.psiH[f.face], f.c0, f.c1, pl,
                                         4 * (b + m) + 2, &full[s]);
                        if constexpr (AIR)
                            tma::load_4d(ss + G::sAH, &maps.airH[f.face], f.ca0, f.c1, pl, 2, &full[s]);
                    }
                }
            }
            flags[1] = t;
        }
    } else {
        // compute warps: TJ per field set; in field set m = warp / TJ, owned
        // cell (row warp % TJ, lane), and halo cell x for the set's first NX
        // threads (row TJ, then column TK)
        const int m = warp / TJ, row = warp % TJ, lt = tid - 32 * TJ * m;
        const long long fs = 3 * g.vol * (long long)(b + m);
        T* __restrict__ Eg = p.e_next + fs;
        T* __restrict__ Hg = p.h_next + fs;
        const int jo = j0 + row, ko = k0 + lane;
        const bool v_own = jo <= g.ny && ko <= g.nz;
        const bool has_x = lt < NX;
        const int rx = lt <= TK ? TJ : lt - TK - 1;
        const int cx = lt <= TK ? lt : TK;
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
                T* en = ring + ((t % 3) * NB + m) * 3 * G::cN;
                step_E<T, TJ, NS, NSLOT, AIR, CK, NB>(p, sl, st, stp, m, en, row, lane, i, jo, ko, v_own && i < i1, Eg);
                if (has_x)
                    step_E<T, TJ, NS, NSLOT, AIR, CK, NB>(p, sl, st, stp, m, en, rx, cx, i, jx, kx, own_x && i < i1,
                                                          Eg);
            }
            tma::compute_barrier(NC);
            if (flags[0]) {
                if (tid == 0) flags[2] = t;
                break;
            }
            if (t > 1) {
                const unsigned char* stp = smem + ((t - 1) % NS) * G::stage;
                const T* enp = ring + (((t - 1) % 3) * NB + m) * 3 * G::cN;
                const T* enc = ring + ((t % 3) * NB + m) * 3 * G::cN;
                if (v_own)
                    step_H<T, TJ, NS, NSLOT, AIR, CK, NB, false>(p, sl, stp, m, enp, enc, row, lane, i - 1, jo, ko, Hg);
                if (own_x)
                    step_H<T, TJ, NS, NSLOT, AIR, CK, NB, true>(p, sl, stp, m, enp, enc, rx, cx, i - 1, jx, kx, Hg);
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

// ---------------------------------------------------------------------------
// Dead-unit skipping (reference: solver/_tile_skip.py:187-285,
// build_tile_skip_plan).  An E edge is dead when alpha_E = beta_E = 0 (the
// update writes +0 forever); an H face is skippable when alpha_H = 1 and
// beta_H = 0 (h = h) or when it is curl-dead (its four bounding E edges are
// dead, so curl E = +0 forever); the padding entries of the layout (zero
// coefficients, held at +0) count as both.  A unit all of whose cells are
// dead or skippable, over its rows j0 .. j0+TJ, columns k0 .. k0+TK and
// planes i0 .. i1 (its own cells with the halo row, column and plane: a
// conservative superset), is left out of the launch lists.

__device__ __forceinline__ bool e_dead(const float* a, const float* b, long long o) {
    return a[o] == 0.0f && b[o] == 0.0f;
}
__device__ __forceinline__ bool e_dead(const double* a, const double* b, long long o) {
    return a[o] == 0.0 && b[o] == 0.0;
}

// flags[u] = 1 when unit u (of `units`) has a live cell.
template <typename T>
__global__ void k_unit_live(Geom g, const T* __restrict__ aE, const T* __restrict__ bE, const T* __restrict__ aH,
                            const T* __restrict__ bH, int tj, int ichunk, const int4* __restrict__ units, int* flags) {
    const int4 u = units[blockIdx.x];
    const int k0 = (u.x & 0xffff) * TK, j0 = (u.x >> 16) * tj, i0 = u.y;
    // real cells only (i <= nx, j <= ny, k <= nz): their +1 neighbours stay
    // inside the padded box
    const int nk = min(k0 + TK, g.nz) - k0 + 1, nj = min(j0 + tj, g.ny) - j0 + 1;
    const int ni = min(u.z, g.nx) - i0 + 1;
    const long long vol = g.vol, si = g.si, sj = g.sj;
    bool live = false;
    for (int t = threadIdx.x; t < ni * nj * nk && !live; t += blockDim.x) {
        const int k = k0 + t % nk, j = j0 + (t / nk) % nj, i = i0 + t / (nk * nj);
        const long long o = pidx(g, i, j, k);
        // E: every component dead
        for (int c = 0; c < 3; ++c) live |= !e_dead(aE + c * vol, bE + c * vol, o);
        // H: every component a no-op or curl-dead
        const T* ax = aH;
        const T* bx = bH;
        const bool dEx = e_dead(aE, bE, o), dEy = e_dead(aE + vol, bE + vol, o), dEz = e_dead(aE + 2 * vol, bE + 2 * vol, o);
        const bool curl_dead[3] = {
            dEy && e_dead(aE + vol, bE + vol, o + 1) && dEz && e_dead(aE + 2 * vol, bE + 2 * vol, o + sj),
            dEz && e_dead(aE + 2 * vol, bE + 2 * vol, o + si) && dEx && e_dead(aE, bE, o + 1),
            dEx && e_dead(aE, bE, o + sj) && dEy && e_dead(aE + vol, bE + vol, o + si)};
        for (int c = 0; c < 3; ++c) {
            const T a = ax[c * vol + o], bb = bx[c * vol + o];
            // h = h, or h = 0 (zero coefficients: a padding entry)
            const bool fixed = bb == T(0) && (a == T(1) || a == T(0));
            live |= !(fixed || curl_dead[c]);
        }
    }
    live = __syncthreads_or(live);
    if (threadIdx.x == 0) flags[blockIdx.x] = live ? 1 : 0;
}

// Both buffer sets of the skipped units' own cells made equal to what the
// dense step keeps there: E (all dead) = +0, a curl-dead H = +0, a no-op H
// = its current value (the reference zeroes the provably-zero entries once
// before the march, _tile_skip.py dead_zero_idx_E / _H).
template <typename T>
__global__ void k_dead_units_sync(Geom g, const T* __restrict__ aH, const T* __restrict__ bH, int tj, int ichunk,
                                  const int4* __restrict__ units, T* e_cur, T* h_cur, T* e_oth, T* h_oth) {
    const int4 u = units[blockIdx.x];
    const int b = blockIdx.y;
    const int k0 = (u.x & 0xffff) * TK, j0 = (u.x >> 16) * tj, i0 = u.y;
    // own rows / columns, with the last row / column a tile absorbs
    const int k1 = (k0 + TK == g.nz) ? g.nz + 1 : min(k0 + TK, g.nz + 1);
    const int j1 = (j0 + tj == g.ny) ? g.ny + 1 : min(j0 + tj, g.ny + 1);
    const int i1 = u.z;
    const int nk = k1 - k0, nj = j1 - j0, ni = i1 - i0;
    if (nk <= 0 || nj <= 0 || ni <= 0) return;
    const long long vol = g.vol, fs = 3 * vol * (long long)b;
    for (int t = threadIdx.x; t < ni * nj * nk; t += blockDim.x) {
        const int k = k0 + t % nk, j = j0 + (t / nk) % nj, i = i0 + t / (nk * nj);
        const long long o = pidx(g, i, j, k);
        for (int c = 0; c < 3; ++c) {
            const long long q = fs + c * vol + o;
            e_cur[q] = T(0);
            e_oth[q] = T(0);
            const bool noop = aH[c * vol + o] == T(1) && bH[c * vol + o] == T(0);
            const T v = noop ? h_cur[q] : T(0);  // curl-dead or zero coefficients: +0
            h_cur[q] = v;
            h_oth[q] = v;
        }
    }
}

constexpr size_t kMaxSmemOptin = 232448;  // B200 opt-in per CTA (227 KB), when the device cannot be queried

// An instance is built only when its shared memory fits one CTA.  Every
// variant has its 0-3 slot instances; a six-slot one (both faces of an axis
// reaching one unit: small grids) may be missing, and a plan that needs it
// is refused when the units are planned.
template <typename T, int TJ, int NS, int NSLOT, bool AIR, int CK, int NB>
constexpr bool slab_fits() {
    return SlabGeo<T, TJ, NS, NSLOT, AIR, CK, NB>::smem <= kMaxSmemOptin;
}

// Slab variants: (TJ, NS of the CPML-free list, NS of the CPML lists, NB
// field sets per CTA).
template <typename F>
bool slab_dispatch(int variant, F&& f) {
    switch (variant) {
        case 0: f.template run<4, 3, 3, 1>(); return true;
        case 1: f.template run<2, 3, 3, 1>(); return true;
        case 2: f.template run<3, 3, 3, 1>(); return true;
        case 3: f.template run<4, 4, 4, 1>(); return true;
        case 4: f.template run<3, 4, 4, 1>(); return true;
        case 5: f.template run<2, 4, 4, 1>(); return true;
        case 6: f.template run<8, 3, 3, 1>(); return true;
        case 7: f.template run<6, 3, 3, 1>(); return true;
        case 8: f.template run<4, 3, 3, 2>(); return true;
        case 9: f.template run<4, 3, 3, 4>(); return true;
        default: return false;
    }
}

template <typename T, int TJ, int NS, int NSLOT, bool AIR, int CK, int NB, typename G>
void one_if_fits(G&& g) {
    if constexpr (slab_fits<T, TJ, NS, NSLOT, AIR, CK, NB>()) g.template one<T, TJ, NS, NSLOT, AIR, CK, NB>();
}

// Every kernel instance of one (TJ, NS, NB) and coefficient storage CK: slot
// capacities 0, 1, 2, 3, 6, with and without air masks.
template <typename T, int TJ, int NS, int CK, int NB, typename G>
void each_instance_ck(G&& g) {
    one_if_fits<T, TJ, NS, 0, false, CK, NB>(g);
    one_if_fits<T, TJ, NS, 1, false, CK, NB>(g);
    one_if_fits<T, TJ, NS, 2, false, CK, NB>(g);
    one_if_fits<T, TJ, NS, 3, false, CK, NB>(g);
    one_if_fits<T, TJ, NS, 6, false, CK, NB>(g);
    one_if_fits<T, TJ, NS, 1, true, CK, NB>(g);
    one_if_fits<T, TJ, NS, 2, true, CK, NB>(g);
    one_if_fits<T, TJ, NS, 3, true, CK, NB>(g);
    one_if_fits<T, TJ, NS, 6, true, CK, NB>(g);
}

// All instances of one (TJ, NS, NB): native coefficients, and float16
// storage for float32 fields.
template <typename T, int TJ, int NS, int NB, typename G>
void each_instance(G&& g) {
    each_instance_ck<T, TJ, NS, kCoefNative, NB>(g);
    if constexpr (sizeof(T) == 4) each_instance_ck<T, TJ, NS, kCoefF16, NB>(g);
}

struct Prepare {
    cudaError_t err = cudaSuccess;
    template <typename T, int TJ, int NS, int NSLOT, bool AIR, int CK, int NB>
    void one() {
        const cudaError_t e = cudaFuncSetAttribute(k_step_slab<T, TJ, NS, NSLOT, AIR, CK, NB>,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)SlabGeo<T, TJ, NS, NSLOT, AIR, CK, NB>::smem);
        if (err == cudaSuccess) err = e;
    }
};

// Shape of a variant: tile rows, field sets per CTA, the largest shared
// memory of the instances every plan needs (0-3 slots, native coefficients:
// the float16 boxes are smaller), whether the six-slot instances exist, and
// the occupancy of the CPML-free instance.
template <typename T>
struct SlabInfo {
    size_t smem = 0;
    int tj = 0, nb = 1, occ0 = 1;
    bool six = false, six_air = false;
    template <int TJ, int NS, int NSC, int NB>
    void run() {
        constexpr int CK = kCoefNative;
        smem = std::max({SlabGeo<T, TJ, NS, 0, false, CK, NB>::smem, SlabGeo<T, TJ, NSC, 3, false, CK, NB>::smem,
                         SlabGeo<T, TJ, NSC, 3, true, CK, NB>::smem});
        six = slab_fits<T, TJ, NSC, 6, false, CK, NB>();
        six_air = slab_fits<T, TJ, NSC, 6, true, CK, NB>();
        tj = TJ;
        nb = NB;
        if constexpr (slab_fits<T, TJ, NS, 0, false, CK, NB>())
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ0, k_step_slab<T, TJ, NS, 0, false, CK, NB>,
                                                          32 * (TJ * NB + 1), SlabGeo<T, TJ, NS, 0, false, CK, NB>::smem);
    }
};

template <typename T>
struct SlabPrepare {
    cudaError_t err = cudaSuccess;
    template <int TJ, int NS, int NSC, int NB>
    void run() {
        Prepare pr;
        each_instance<T, TJ, NS, NB>(pr);
        if constexpr (NSC != NS) each_instance<T, TJ, NSC, NB>(pr);
        err = pr.err;
    }
};

template <typename T>
struct SlabLaunch {
    const SlabMaps& m;
    const StencilArgs<T>& a;
    const int4* const* units;
    const int* n_units;
    bool air;
    int* status;
    const cudaStream_t* streams;  // one per list
    int launched = 0;
    bool missing = false;  // a list whose instance is not built (refused when planned)
    int priority = 0;      // scheduling priority of the CPML lists' CTAs (0: the default)
    template <int NSLOT, bool AIR, int CK, int TJ, int NS, int NB>
    void go(int q) {
        if (n_units[q] <= 0) return;
        if constexpr (slab_fits<T, TJ, NS, NSLOT, AIR, CK, NB>()) {
            cudaLaunchConfig_t cfg{};
            cfg.gridDim = dim3((unsigned)n_units[q] * (a.B / NB));
            cfg.blockDim = dim3(32 * (TJ * NB + 1));
            cfg.dynamicSmemBytes = SlabGeo<T, TJ, NS, NSLOT, AIR, CK, NB>::smem;
            cfg.stream = streams[q];
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributePriority;
            at[0].val.priority = q > 0 ? priority : 0;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            cudaLaunchKernelEx(&cfg, k_step_slab<T, TJ, NS, NSLOT, AIR, CK, NB>, m, a, units[q], status);
            ++launched;
        } else {
            missing = true;
        }
    }
    template <int CK, int TJ, int NS, int NSC, int NB>
    void run_ck() {
        // the CPML lists first: their units march longer chains, the
        // CPML-free list fills the SMs around them
        if (order_cpml_first) {
            // most slots (the longest marches) first
            go_air<6, CK, TJ, NSC, NB>(4);
            go_air<3, CK, TJ, NSC, NB>(3);
            go_air<2, CK, TJ, NSC, NB>(2);
            go_air<1, CK, TJ, NSC, NB>(1);
            go<0, false, CK, TJ, NS, NB>(0);
            return;
        }
        go<0, false, CK, TJ, NS, NB>(0);
        go_air<1, CK, TJ, NSC, NB>(1);
        go_air<2, CK, TJ, NSC, NB>(2);
        go_air<3, CK, TJ, NSC, NB>(3);
        go_air<6, CK, TJ, NSC, NB>(4);
    }
    bool order_cpml_first = false;
    template <int NSLOT, int CK, int TJ, int NS, int NB>
    void go_air(int q) {
        if (air)
            go<NSLOT, true, CK, TJ, NS, NB>(q);
        else
            go<NSLOT, false, CK, TJ, NS, NB>(q);
    }
    template <int TJ, int NS, int NSC, int NB>
    void run() {
        if (a.B % NB != 0) {
            missing = true;
            return;
        }
        if constexpr (sizeof(T) == 4) {
            if (a.coef_kind == kCoefF16) {
                run_ck<kCoefF16, TJ, NS, NSC, NB>();
                return;
            }
        }
        run_ck<kCoefNative, TJ, NS, NSC, NB>();
    }
};


}  // namespace

int slab_tj_of(int variant) {
    SlabInfo<float> f;
    if (!slab_dispatch(variant, f)) return 0;
    return f.tj;
}

int slab_nb_of(int variant) {
    SlabInfo<float> f;
    if (!slab_dispatch(variant, f)) return 1;
    return f.nb;
}

template <typename T>
bool slab_six_ok(int variant, bool air) {
    SlabInfo<T> f;
    if (!slab_dispatch(variant, f)) return false;
    return air ? f.six_air : f.six;
}
template bool slab_six_ok<float>(int, bool);
template bool slab_six_ok<double>(int, bool);

template <typename T>
bool slab_supported(int variant) {
    SlabInfo<T> f;
    if (!slab_dispatch(variant, f)) return false;
    int dev = 0, optin = 0;
    size_t limit = kMaxSmemOptin;
    if (cudaGetDevice(&dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) == cudaSuccess && optin > 0)
        limit = (size_t)optin;
    return f.smem <= limit;
}
template bool slab_supported<float>(int);
template bool slab_supported<double>(int);

template <typename T>
cudaError_t prepare_slab(int variant) {
    SlabPrepare<T> f;
    if (!slab_dispatch(variant, f)) return cudaErrorInvalidValue;
    return f.err;
}
template cudaError_t prepare_slab<float>(int);
template cudaError_t prepare_slab<double>(int);

template <typename T>
int slab_occupancy(int variant) {
    SlabInfo<T> f;
    slab_dispatch(variant, f);
    return f.occ0 < 1 ? 1 : f.occ0;
}
template int slab_occupancy<float>(int);
template int slab_occupancy<double>(int);

// Chunks [i0, i1) of the i march: about `ichunk` planes each, cut at the
// x faces' slab boundaries so that a chunk either holds a slab's planes or
// none of them (E_new(i1) is part of a chunk's work, so a chunk ending at
// i1 = lo - 1 stays clear of a slab starting at lo), with no chunk shorter
// than four planes (a short piece joins its neighbour).
std::vector<int2> slab_chunks(const Geom& g, const FaceDev* f, int nfaces, int ichunk) {
    const int nplanes = g.nx + 1;
    std::vector<int> cuts = {0, nplanes};
    for (int q = 0; q < nfaces; ++q) {
        if (f[q].axis != 0) continue;
        for (int c : {f[q].lo - 1, f[q].lo + f[q].n})
            if (c > 0 && c < nplanes) cuts.push_back(c);
    }
    std::sort(cuts.begin(), cuts.end());
    cuts.erase(std::unique(cuts.begin(), cuts.end()), cuts.end());
    std::vector<int> kept = {0};
    for (size_t q = 1; q < cuts.size(); ++q) {
        const bool end = cuts[q] == nplanes;
        if (!end && cuts[q] - kept.back() < 4) continue;
        if (end && kept.size() > 1 && cuts[q] - kept.back() < 4) kept.pop_back();
        kept.push_back(cuts[q]);
    }
    std::vector<int2> out;
    for (size_t q = 0; q + 1 < kept.size(); ++q) {
        const int a = kept[q], b = kept[q + 1];
        const int m = (b - a + ichunk - 1) / ichunk;
        for (int t = 0; t < m; ++t)
            out.push_back(make_int2(a + (int)((long long)(b - a) * t / m), a + (int)((long long)(b - a) * (t + 1) / m)));
    }
    return out;
}

// Units of the slab step, sorted into lists by their number of CPML face
// slots: lists 0-3 hold the units with that many slots, list 4 those with
// four to six (on small grids both faces of an axis can reach one unit; its
// launch has six slots, the unused ones empty).  A unit's E cells span rows
// j0 .. j0+TJ (its own rows and the halo row), columns k0 .. k0+TK and
// planes i0 .. i1 (E_new(i1) feeds H_new(i1-1)); every face whose slab
// meets those ranges on its axis gets a slot, slots in face (boundary)
// order.  A unit is (k tile | j tile << 16, i0, i1, packed slot faces).
// False for more faces than the packed slot indices hold, or tile counts
// beyond the packing.
bool plan_slab_units(const Geom& g, const FaceDev* f, int nfaces, int tj, int ichunk, std::vector<int4> out[5]) {
    for (int q = 0; q < 5; ++q) out[q].clear();
    if (nfaces > kMaxFaces || tj <= 0 || ichunk <= 0) return false;
    const int nkt = g.nz % TK == 0 ? g.nz / TK : (g.nz + TK) / TK;
    const int njt = g.ny % tj == 0 ? g.ny / tj : (g.ny + tj) / tj;
    if (nkt > 0xffff || njt > 0x7fff) return false;
    const std::vector<int2> chunks = slab_chunks(g, f, nfaces, ichunk);
    const int nch = (int)chunks.size();
    // bit mask of the faces of `axis` whose slab [lo_f, lo_f + n) meets [lo, hi]
    auto faces_on = [&](int axis, int lo, int hi) {
        unsigned m = 0;
        for (int q = 0; q < nfaces; ++q)
            if (f[q].axis == axis && f[q].lo <= hi && f[q].lo + f[q].n - 1 >= lo) m |= 1u << q;
        return m;
    };
    std::vector<unsigned> fk(nkt), fj(njt), fi(nch);
    for (int t = 0; t < nkt; ++t) fk[t] = faces_on(2, t * TK, t * TK + TK);
    for (int t = 0; t < njt; ++t) fj[t] = faces_on(1, t * tj, t * tj + tj);
    for (int c = 0; c < nch; ++c) fi[c] = faces_on(0, chunks[c].x, chunks[c].y);
    for (int c = 0; c < nch; ++c)
        for (int jt = 0; jt < njt; ++jt)
            for (int kt = 0; kt < nkt; ++kt) {
                const unsigned m = fi[c] | fj[jt] | fk[kt];
                const int ns = __builtin_popcount(m);
                const int list = ns <= 3 ? ns : 4;  // capacities 0, 1, 2, 3, 6
                const int cap = ns <= 3 ? ns : kSlotMax;
                int w = 0, q = 0;
                for (int fq = 0; fq < nfaces; ++fq)  // ascending: boundary order
                    if (m >> fq & 1) w |= fq << (4 * q++);
                for (; q < cap; ++q) w |= 15 << (4 * q);  // empty slots
                out[list].push_back(make_int4(kt | (jt << 16), chunks[c].x, chunks[c].y, w));
            }
    return true;
}

template <typename T>
int slab_unit_liveness(const Geom& g, const T* aE, const T* bE, const T* aH, const T* bH, int tj, int ichunk,
                       const int4* units, int n, int* flags, cudaStream_t s) {
    if (n <= 0) return 0;
    k_unit_live<T><<<n, 256, 0, s>>>(g, aE, bE, aH, bH, tj, ichunk, units, flags);
    return 1;
}
template int slab_unit_liveness<float>(const Geom&, const float*, const float*, const float*, const float*, int, int,
                                       const int4*, int, int*, cudaStream_t);
template int slab_unit_liveness<double>(const Geom&, const double*, const double*, const double*, const double*, int,
                                        int, const int4*, int, int*, cudaStream_t);

template <typename T>
int slab_dead_sync(const Geom& g, const T* aH, const T* bH, int tj, int ichunk, const int4* units, int n, int B,
                   T* e_cur, T* h_cur, T* e_oth, T* h_oth, cudaStream_t s) {
    if (n <= 0) return 0;
    k_dead_units_sync<T><<<dim3(n, B), 256, 0, s>>>(g, aH, bH, tj, ichunk, units, e_cur, h_cur, e_oth, h_oth);
    return 1;
}
template int slab_dead_sync<float>(const Geom&, const float*, const float*, int, int, const int4*, int, int, float*,
                                   float*, float*, float*, cudaStream_t);
template int slab_dead_sync<double>(const Geom&, const double*, const double*, int, int, const int4*, int, int,
                                    double*, double*, double*, double*, cudaStream_t);

template <typename T>
StreamPlan plan_slab(const Geom& g, int sm_count, int ctas_per_sm, int B, int variant) {
    SlabInfo<T> f;
    slab_dispatch(variant, f);
    StreamPlan s{};
    s.block_y = f.tj;
    s.grid_x = (g.nz % TK == 0 ? g.nz / TK : (g.nz + TK) / TK) * std::max(1, B / f.nb);
    s.grid_y = g.ny % f.tj == 0 ? g.ny / f.tj : (g.ny + f.tj) / f.tj;
    const long long tiles = (long long)s.grid_x * s.grid_y;
    const int nplanes = g.nx + 1;
    const int per_wave = sm_count * ctas_per_sm;
    // chunks of about 16 planes (as the tile step), best wave quantisation
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
template StreamPlan plan_slab<float>(const Geom&, int, int, int, int);
template StreamPlan plan_slab<double>(const Geom&, int, int, int, int);

template <typename T>
int launch_slab_step(StencilArgs<T> a, int ichunk, int variant, const int4* const units[5], const int n_units[5],
                     bool air, int* status, const cudaStream_t streams[5]) {
    SlabInfo<T> info;
    if (!slab_dispatch(variant, info)) return -1;
    const int tj = info.tj, nb = info.nb;
    if (a.B % nb != 0) return -4;
    SlabMaps m;
    const long long nset = 3LL * a.B;
    // E and H boxes: the three components of the CTA's nb field sets
    if (!tma::encode_field_map<T>(&m.e, a.e, a.g, (int)nset, TK + 4, tj + 1, 3 * nb) ||
        !tma::encode_field_map<T>(&m.h, a.h, a.g, (int)nset, TK + 8, tj + 2, 3 * nb))
        return -2;
    if (a.coef_kind == kCoefF16) {
        // 16-bit coefficient boxes: E rows of 40 entries (80 bytes), H rows of 32
        if (sizeof(T) != 4 || (a.g.nkp * 2) % 16 != 0) return -3;
        const unsigned long long dims[4] = {(unsigned long long)a.g.nkp, (unsigned long long)a.g.njp,
                                            (unsigned long long)(a.g.nx + 4), 3ULL};
        const unsigned long long str[3] = {(unsigned long long)a.g.sj * 2, (unsigned long long)a.g.si * 2,
                                           (unsigned long long)a.g.vol * 2};
        const unsigned bE_[4] = {40u, (unsigned)(tj + 1), 1, 3}, bH_[4] = {(unsigned)TK, (unsigned)tj, 1, 3};
        const CUtensorMapDataType u16 = CU_TENSOR_MAP_DATA_TYPE_UINT16;
        if (!tma::encode_4d(&m.aE, u16, a.cq[0], dims, str, bE_) || !tma::encode_4d(&m.bE, u16, a.cq[1], dims, str, bE_) ||
            !tma::encode_4d(&m.aH, u16, a.cq[2], dims, str, bH_) || !tma::encode_4d(&m.bH, u16, a.cq[3], dims, str, bH_))
            return -2;
    } else if (!tma::encode_field_map<T>(&m.aE, a.aE, a.g, 3, TK + 4, tj + 1) ||
               !tma::encode_field_map<T>(&m.bE, a.bE, a.g, 3, TK + 4, tj + 1) ||
               !tma::encode_field_map<T>(&m.aH, a.aH, a.g, 3, TK, tj) ||
               !tma::encode_field_map<T>(&m.bH, a.bH, a.g, 3, TK, tj)) {
        return -2;
    }
    const CUtensorMapDataType dt = sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    for (int q = 0; q < a.nfaces; ++q) {
        const FaceDev& f = a.f[q];
        // psi: (entry, row, plane, component) over [B][4][slab]; air: [4][slab] bytes
        const unsigned long long pd[4] = {(unsigned long long)f.dK, (unsigned long long)f.dJ,
                                          (unsigned long long)f.dI, 4ULL * a.B};
        const unsigned long long ps[3] = {(unsigned long long)f.pk * sizeof(T),
                                          (unsigned long long)f.pk * f.dJ * sizeof(T),
                                          (unsigned long long)f.slab * sizeof(T)};
        const unsigned long long ad[4] = {(unsigned long long)f.dK, (unsigned long long)f.dJ,
                                          (unsigned long long)f.dI, 4ULL};
        const unsigned long long as[3] = {(unsigned long long)f.pk, (unsigned long long)f.pk * f.dJ,
                                          (unsigned long long)f.slab};
        const unsigned bpE[4] = {(unsigned)PW, (unsigned)(tj + 1), 1, 2}, bpH[4] = {(unsigned)PW, (unsigned)tj, 1, 2};
        const unsigned baE[4] = {(unsigned)AW, (unsigned)(tj + 1), 1, 2}, baH[4] = {(unsigned)AW, (unsigned)tj, 1, 2};
        if (!tma::encode_4d(&m.psiE[q], dt, f.psi, pd, ps, bpE) || !tma::encode_4d(&m.psiH[q], dt, f.psi, pd, ps, bpH) ||
            !tma::encode_4d(&m.airE[q], CU_TENSOR_MAP_DATA_TYPE_UINT8, f.air, ad, as, baE) ||
            !tma::encode_4d(&m.airH[q], CU_TENSOR_MAP_DATA_TYPE_UINT8, f.air, ad, as, baH))
            return -2;
    }
    a.ichunk = ichunk;
    SlabLaunch<T> l{m, a, units, n_units, air, status, streams};
    // The CPML lists are launched first (most slots first) and their CTAs
    // scheduled at the highest priority, so their longer marches start
    // early and the CPML-free list fills the SMs around them: measured on
    // the 256^3 brick box, the slab step from 0.422 to 0.401 ms.  The
    // environment variables FITB_SLAB_ORDER=free_first and
    // FITB_SLAB_PRIORITY=0 restore the plain order and priority (read once
    // per process; tuning switches, every setting computes the same bits).
    static const bool cpml_first = [] {
        const char* e = std::getenv("FITB_SLAB_ORDER");
        return !(e && !std::strcmp(e, "free_first"));
    }();
    static const int high = [] {
        const char* e = std::getenv("FITB_SLAB_PRIORITY");
        int lo = 0, hi = 0;
        if ((e && std::atoi(e) == 0) || cudaDeviceGetStreamPriorityRange(&lo, &hi) != cudaSuccess) return 0;
        return hi;  // numerically lowest: the highest priority
    }();
    l.order_cpml_first = cpml_first;
    l.priority = high;
    slab_dispatch(variant, l);
    return l.missing ? -4 : l.launched;
}
template int launch_slab_step<float>(StencilArgs<float>, int, int, const int4* const[5], const int[5], bool, int*,
                                     const cudaStream_t[5]);
template int launch_slab_step<double>(StencilArgs<double>, int, int, const int4* const[5], const int[5], bool, int*,
                                      const cudaStream_t[5]);

}  // namespace fitb
