// One leapfrog step (E update, then H update) in a single pass over the
// grid: the fused i-march.
//
// Same arithmetic as the two-pass kernels (reference: numba_kernels.py:36-127
// for the curl updates, cpml.py:343-516 for the psi recursion and its
// correction); the step reads E, H and psi from one buffer set and writes
// the new values to the other (the handle swaps them every step), so a CTA
// never sees a neighbour's new values where it needs old ones.
//
// Work mapping: a CTA is 32 lanes along k by TJ warps along j and marches
// over a chunk [i0, i1) of i planes.  At plane i a thread computes E_new(i)
// of its cell (H_old at i-1 from registers, at j-1 by a load that the row
// above has brought into L1, at k-1 by a warp shuffle) and then H_new(i-1)
// (E_new at i from registers, at k+1 by a warp shuffle, at j+1 from the
// next warp through shared memory).  The last lane and the last warp
// compute E_new only as neighbours of the others' H: tiles overlap by one
// column and one row, and those cells are stored by the neighbouring tile.
// A chunk also computes E_new at its plane i1 (not stored) for H_new(i1-1).
// One __syncthreads per plane orders the shared-memory exchange (written
// after the reads of the same plane, double-buffered across planes).
//
// Ports write E between the E and the H update (operator.py:1351-1536,
// lumped operator.py:134-166).  The H cells whose curl takes a port-written
// E edge are recomputed afterwards from the old buffers by k_fix_H with the
// same arithmetic (H_old, psi_old are still intact in the other buffers).
#include "fused_cpml.cuh"

namespace fitb {

namespace {

// Everything a thread loads for one plane.
template <typename T>
struct FPlane {
    T ex, ey, ez;             // E_old of the cell
    T hx, hy, hz;             // H_old of the cell
    T hz_jm, hx_jm;           // H_old at j-1
    T hy_before, hx_before;   // H_old at k-1 (lane 0 only)
    FCoef<T> ce, ch;          // alpha/beta of E and of H
};

template <typename T>
__device__ __forceinline__ void load_plane(FPlane<T>& q, const StencilArgs<T>& p, const T* __restrict__ E,
                                           const T* __restrict__ H, long long o, bool lane0) {
    const long long vol = p.g.vol, sj = p.g.sj;
    q.ex = __ldg(E + o);
    q.ey = __ldg(E + vol + o);
    q.ez = __ldg(E + 2 * vol + o);
    q.hx = __ldg(H + o);
    q.hy = __ldg(H + vol + o);
    q.hz = __ldg(H + 2 * vol + o);
    q.hz_jm = __ldg(H + 2 * vol + o - sj);
    q.hx_jm = __ldg(H + o - sj);
    q.hy_before = lane0 ? __ldg(H + vol + o - 1) : T(0);
    q.hx_before = lane0 ? __ldg(H + o - 1) : T(0);
    load_coef3(q.ce, p.aE, p.bE, o, vol);
    load_coef3(q.ch, p.aH, p.bH, o, vol);
}

constexpr unsigned kAll = 0xffffffffu;

template <typename T, int TJ>
__global__ void __launch_bounds__(32 * TJ) k_step_fused(const StencilArgs<T> p) {
    const Geom& g = p.g;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int ntj = (g.ny + TJ - 1) / (TJ - 1);  // j tiles: ceil((ny + 1) / (TJ - 1))
    const int b = blockIdx.y / ntj;
    const int k = blockIdx.x * 31 + lane;
    const int j = (blockIdx.y - b * ntj) * (TJ - 1) + w;
    // loads stay inside the padded plane; clamped threads compute values
    // that no owned cell uses
    const int kl = min(k, g.nkp - 1), jl = min(j, g.njp - 1);
    const bool cell = k <= g.nz && j <= g.ny;
    const bool own = cell && lane < 31 && w < TJ - 1;
    const int i0 = blockIdx.z * p.ichunk;
    const int i1 = min(i0 + p.ichunk, g.nx + 1);
    const long long vol = g.vol, si = g.si, fs = 3 * vol;
    const T* __restrict__ E = p.e + b * fs;
    const T* __restrict__ H = p.h + b * fs;
    T* __restrict__ En = p.e_next + b * fs;
    T* __restrict__ Hn = p.h_next + b * fs;
    const unsigned mjk = cell ? mask_jk(p, j, k) : 0u;
    __shared__ T s_ex[2][TJ][32];
    __shared__ T s_ez[2][TJ][32];
    const int wn = w + 1 < TJ ? w + 1 : w;

    long long o = (long long)(i0 + 2) * si + (long long)jl * g.sj + kl;
    T hz_im = __ldg(H + 2 * vol + o - si);
    T hy_im = __ldg(H + vol + o - si);
    FPlane<T> cur, nxt;
    load_plane(cur, p, E, H, o, lane == 0);
    // plane i-1 state for its H update
    T ex_p = T(0), ey_p = T(0), ez_p = T(0), hx_p = T(0), hy_p = T(0), hz_p = T(0);
    FCoef<T> ch_p = cur.ch;
    for (int i = i0; i <= i1; ++i) {
        if (i < i1) load_plane(nxt, p, E, H, o + si, lane == 0);
        // j+1 neighbours of E_new(i-1), written by the next warp last plane
        T ez_jp = T(0), ex_jp = T(0);
        if (i > i0) {
            ez_jp = s_ez[(i - 1) & 1][wn][lane];
            ex_jp = s_ex[(i - 1) & 1][wn][lane];
        }
        // ---- E_new(i) ----
        const T hy_up = __shfl_up_sync(kAll, cur.hy, 1);
        const T hx_up = __shfl_up_sync(kAll, cur.hx, 1);
        const T hy_km = lane == 0 ? cur.hy_before : hy_up;
        const T hx_km = lane == 0 ? cur.hx_before : hx_up;
        const T cxe = ((cur.hz - cur.hz_jm) - cur.hy) + hy_km;
        const T cye = ((cur.hx - hx_km) - cur.hz) + hz_im;
        const T cze = ((cur.hy - hy_im) - cur.hx) + cur.hx_jm;
        T ex_n = cur.ce.ax * cur.ex + cur.ce.bx * cxe;
        T ey_n = cur.ce.ay * cur.ey + cur.ce.by * cye;
        T ez_n = cur.ce.az * cur.ez + cur.ce.bz * cze;
        const bool e_store = own && i < i1;
        const unsigned me = (cell && i <= g.nx) ? (mjk | mask_i(p, i)) : 0u;
        if (me)
            cpml_E(p, me, b, i, j, k, cur.hz - hz_im, cur.hy - hy_im, cur.hz - cur.hz_jm, cur.hx - cur.hx_jm,
                   cur.hy - hy_km, cur.hx - hx_km, cur.ce, ex_n, ey_n, ez_n, e_store);
        if (e_store) {
            En[o] = ex_n;
            En[vol + o] = ey_n;
            En[2 * vol + o] = ez_n;
        }
        // ---- H_new(i-1) ----
        const T ey_dn = __shfl_down_sync(kAll, ey_p, 1);
        const T ex_dn = __shfl_down_sync(kAll, ex_p, 1);
        if (i > i0 && own) {
            const T ey_kp = ey_dn, ex_kp = ex_dn;
            const T cxh = ((ez_jp - ez_p) - ey_kp) + ey_p;
            const T cyh = ((ex_kp - ex_p) - ez_n) + ez_p;
            const T czh = ((ey_n - ey_p) - ex_jp) + ex_p;
            T hx_n = ch_p.ax * hx_p - ch_p.bx * cxh;
            T hy_n = ch_p.ay * hy_p - ch_p.by * cyh;
            T hz_n = ch_p.az * hz_p - ch_p.bz * czh;
            const unsigned mh = mjk | mask_i(p, i - 1);
            if (mh)
                cpml_H(p, mh, b, i - 1, j, k, ez_n - ez_p, ey_n - ey_p, ez_jp - ez_p, ex_jp - ex_p, ey_kp - ey_p,
                       ex_kp - ex_p, ch_p, hx_n, hy_n, hz_n);
            const long long oh = o - si;
            Hn[oh] = hx_n;
            Hn[vol + oh] = hy_n;
            Hn[2 * vol + oh] = hz_n;
        }
        s_ex[i & 1][w][lane] = ex_n;
        s_ez[i & 1][w][lane] = ez_n;
        __syncthreads();
        ex_p = ex_n;
        ey_p = ey_n;
        ez_p = ez_n;
        hx_p = cur.hx;
        hy_p = cur.hy;
        hz_p = cur.hz;
        ch_p = cur.ch;
        hz_im = cur.hz;
        hy_im = cur.hy;
        cur = nxt;
        o += si;
    }
}

// H update of listed cells, from the old H / psi buffers and the current
// (port-written) E: the fused step's H at cells next to port edges.
template <typename T>
__global__ void k_fix_H(const StencilArgs<T> p, const int4* __restrict__ cells, int n) {
    const Geom& g = p.g;
    const long long vol = g.vol, si = g.si, sj = g.sj, fs = 3 * vol;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)n * p.B;
         t += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(t / n);
        const int4 c = cells[t - (long long)b * n];
        const int i = c.x, j = c.y, k = c.z;
        const T* E = p.e_next + b * fs;
        const T* Hold = p.h + b * fs;
        T* Hn = p.h_next + b * fs;
        const long long o = pidx(g, i, j, k);
        const T ex = E[o], ey = E[vol + o], ez = E[2 * vol + o];
        const T ez_jp = E[2 * vol + o + sj], ex_jp = E[o + sj];
        const T ey_kp = E[vol + o + 1], ex_kp = E[o + 1];
        const T ez_ip = E[2 * vol + o + si], ey_ip = E[vol + o + si];
        FCoef<T> ch;
        load_coefH_stored(ch, p, o, vol);  // the storage the step kernel read
        const T cxh = ((ez_jp - ez) - ey_kp) + ey;
        const T cyh = ((ex_kp - ex) - ez_ip) + ez;
        const T czh = ((ey_ip - ey) - ex_jp) + ex;
        T hx_n = ch.ax * Hold[o] - ch.bx * cxh;
        T hy_n = ch.ay * Hold[vol + o] - ch.by * cyh;
        T hz_n = ch.az * Hold[2 * vol + o] - ch.bz * czh;
        const unsigned mh = mask_jk(p, j, k) | mask_i(p, i);
        if (mh)
            cpml_H(p, mh, b, i, j, k, ez_ip - ez, ey_ip - ey, ez_jp - ez, ex_jp - ex, ey_kp - ey, ex_kp - ex, ch,
                   hx_n, hy_n, hz_n);
        Hn[o] = hx_n;
        Hn[vol + o] = hy_n;
        Hn[2 * vol + o] = hz_n;
    }
}

// ---------------------------------------------------------------------------
// Shared-memory pipelined form of the fused step.  The planes a CTA needs
// are staged by cp.async (4- or 8-byte copies, one per element, no register
// cost) NS-1 planes ahead of the plane being computed; a stage holds for one
// plane: H_old on rows j0-1 .. j0+TJ-1 and columns k0-1 .. k0+31 (the j-1
// and k-1 halos of the E update), E_old and the twelve coefficient arrays on
// the TJ x 32 tile.  cp.async.wait_group and one __syncthreads per plane
// order the copies (no polling loop).  The j+1 exchange of E_new goes
// through a separate double buffer as in the register form.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void cp_async_el(T* smem, const T* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    if constexpr (sizeof(T) == 4)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// CS: the coefficients go through the stages too (else each thread
// prefetches its own twelve one plane ahead in registers).
template <int TJ, bool CS>
struct PipeLayout {
    static constexpr int kHc = 33;                       // H columns k0-1 .. k0+31
    static constexpr int kHrows = TJ + 1;                // H rows j0-1 .. j0+TJ-1
    static constexpr int kH = 3 * kHrows * kHc;          // H_old
    static constexpr int kTile = TJ * 32;
    static constexpr int kStage = kH + (CS ? 15 : 3) * kTile;  // + E_old (3) [+ aE bE aH bH (12)]
};

template <typename T, int TJ, int NS, bool CS, int MINB>
__global__ void __launch_bounds__(32 * TJ, MINB) k_step_fused_pipe(const StencilArgs<T> p) {
    using L = PipeLayout<TJ, CS>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* stages = reinterpret_cast<T*>(smem_raw);
    T* s_en = stages + NS * L::kStage;  // [2][2][TJ][32]: E_new x and z
    const Geom& g = p.g;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int ntj = (g.ny + TJ - 1) / (TJ - 1);
    const int b = blockIdx.y / ntj;
    const int k = blockIdx.x * 31 + lane;
    const int j = (blockIdx.y - b * ntj) * (TJ - 1) + w;
    const int kl = min(k, g.nkp - 1), jl = min(j, g.njp - 1);
    const bool cell = k <= g.nz && j <= g.ny;
    const bool own = cell && lane < 31 && w < TJ - 1;
    const int i0 = blockIdx.z * p.ichunk;
    const int i1 = min(i0 + p.ichunk, g.nx + 1);
    const long long vol = g.vol, si = g.si, sj = g.sj, fs = 3 * vol;
    const T* __restrict__ E = p.e + b * fs;
    const T* __restrict__ H = p.h + b * fs;
    T* __restrict__ En = p.e_next + b * fs;
    T* __restrict__ Hn = p.h_next + b * fs;
    const T* coef[4] = {p.aE, p.bE, p.aH, p.bH};
    const unsigned mjk = cell ? mask_jk(p, j, k) : 0u;
    const int wn = w + 1 < TJ ? w + 1 : w;
    const long long orow = (long long)jl * sj + kl;  // in-plane offset of the own (clamped) cell

    auto issue = [&](int ip, int st) {
        T* sg = stages + st * L::kStage;
        const long long op = (long long)(ip + 2) * si + orow;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            cp_async_el(sg + (c * L::kHrows + w + 1) * L::kHc + lane + 1, H + c * vol + op);
            if (w == 0) cp_async_el(sg + (c * L::kHrows) * L::kHc + lane + 1, H + c * vol + op - sj);
            if (lane == 0) cp_async_el(sg + (c * L::kHrows + w + 1) * L::kHc, H + c * vol + op - 1);
            cp_async_el(sg + L::kH + c * L::kTile + w * 32 + lane, E + c * vol + op);
        }
        if constexpr (CS) {
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    cp_async_el(sg + L::kH + (3 + 3 * a + c) * L::kTile + w * 32 + lane, coef[a] + c * vol + op);
        }
    };
    // register-prefetched coefficients (CS false): ce/ch of the plane being
    // computed, and of the next one
    FCoef<T> rce{}, rch{}, nce{}, nch{};

    // H_old at plane i0-1 (x-neighbours of the first E plane)
    long long o = (long long)(i0 + 2) * si + orow;
    T hz_im = __ldg(H + 2 * vol + o - si);
    T hy_im = __ldg(H + vol + o - si);
#pragma unroll
    for (int q = 0; q < NS - 1; ++q) {
        if (i0 + q <= i1) issue(i0 + q, (i0 + q) % NS);  // plane ip lives in stage ip % NS
        cp_async_commit();
    }
    T ex_p = T(0), ey_p = T(0), ez_p = T(0), hx_p = T(0), hy_p = T(0), hz_p = T(0);
    FCoef<T> ch_p{};
    if constexpr (!CS) {
        load_coef3(rce, p.aE, p.bE, o, vol);
        load_coef3(rch, p.aH, p.bH, o, vol);
    }
    for (int i = i0; i <= i1; ++i) {
        cp_async_wait<NS - 2>();
        __syncthreads();
        if (i + NS - 1 <= i1) issue(i + NS - 1, (i + NS - 1) % NS);
        cp_async_commit();
        if constexpr (!CS) {
            if (i < i1) {
                load_coef3(nce, p.aE, p.bE, o + si, vol);
                load_coef3(nch, p.aH, p.bH, o + si, vol);
            }
        }
        const T* sg = stages + (i % NS) * L::kStage;
        const T* sh = sg;
        const T* se = sg + L::kH;
        const T* sc = se + 3 * L::kTile;
        const int hown = (w + 1) * L::kHc + lane + 1;
        const T hx = sh[hown], hy = sh[L::kHrows * L::kHc + hown], hz = sh[2 * L::kHrows * L::kHc + hown];
        const T hz_jm = sh[2 * L::kHrows * L::kHc + hown - L::kHc];
        const T hx_jm = sh[hown - L::kHc];
        const T hy_km = sh[L::kHrows * L::kHc + hown - 1];
        const T hx_km = sh[hown - 1];
        const int t = w * 32 + lane;
        FCoef<T> ce, ch;
        if constexpr (CS) {
            ce.ax = sc[t]; ce.ay = sc[L::kTile + t]; ce.az = sc[2 * L::kTile + t];
            ce.bx = sc[3 * L::kTile + t]; ce.by = sc[4 * L::kTile + t]; ce.bz = sc[5 * L::kTile + t];
            ch.ax = sc[6 * L::kTile + t]; ch.ay = sc[7 * L::kTile + t]; ch.az = sc[8 * L::kTile + t];
            ch.bx = sc[9 * L::kTile + t]; ch.by = sc[10 * L::kTile + t]; ch.bz = sc[11 * L::kTile + t];
        } else {
            ce = rce;
            ch = rch;
        }
        // ---- E_new(i) ----
        const T cxe = ((hz - hz_jm) - hy) + hy_km;
        const T cye = ((hx - hx_km) - hz) + hz_im;
        const T cze = ((hy - hy_im) - hx) + hx_jm;
        T ex_n = ce.ax * se[t] + ce.bx * cxe;
        T ey_n = ce.ay * se[L::kTile + t] + ce.by * cye;
        T ez_n = ce.az * se[2 * L::kTile + t] + ce.bz * cze;
        const bool e_store = own && i < i1;
        const unsigned me = (cell && i <= g.nx) ? (mjk | mask_i(p, i)) : 0u;
        if (me)
            cpml_E(p, me, b, i, j, k, hz - hz_im, hy - hy_im, hz - hz_jm, hx - hx_jm, hy - hy_km, hx - hx_km, ce,
                   ex_n, ey_n, ez_n, e_store);
        if (e_store) {
            En[o] = ex_n;
            En[vol + o] = ey_n;
            En[2 * vol + o] = ez_n;
        }
        // ---- H_new(i-1) ----
        const T ey_dn = __shfl_down_sync(kAll, ey_p, 1);
        const T ex_dn = __shfl_down_sync(kAll, ex_p, 1);
        if (i > i0 && own) {
            const T* sp = s_en + ((i - 1) & 1) * 2 * L::kTile;
            const T ex_jp = sp[wn * 32 + lane];
            const T ez_jp = sp[L::kTile + wn * 32 + lane];
            const T ey_kp = ey_dn, ex_kp = ex_dn;
            const T cxh = ((ez_jp - ez_p) - ey_kp) + ey_p;
            const T cyh = ((ex_kp - ex_p) - ez_n) + ez_p;
            const T czh = ((ey_n - ey_p) - ex_jp) + ex_p;
            T hx_n = ch_p.ax * hx_p - ch_p.bx * cxh;
            T hy_n = ch_p.ay * hy_p - ch_p.by * cyh;
            T hz_n = ch_p.az * hz_p - ch_p.bz * czh;
            const unsigned mh = mjk | mask_i(p, i - 1);
            if (mh)
                cpml_H(p, mh, b, i - 1, j, k, ez_n - ez_p, ey_n - ey_p, ez_jp - ez_p, ex_jp - ex_p, ey_kp - ey_p,
                       ex_kp - ex_p, ch_p, hx_n, hy_n, hz_n);
            const long long oh = o - si;
            Hn[oh] = hx_n;
            Hn[vol + oh] = hy_n;
            Hn[2 * vol + oh] = hz_n;
        }
        T* sw = s_en + (i & 1) * 2 * L::kTile;
        sw[t] = ex_n;
        sw[L::kTile + t] = ez_n;
        ex_p = ex_n;
        ey_p = ey_n;
        ez_p = ez_n;
        hx_p = hx;
        hy_p = hy;
        hz_p = hz;
        ch_p = ch;
        hz_im = hz;
        hy_im = hy;
        if constexpr (!CS) {
            rce = nce;
            rch = nch;
        }
        o += si;
    }
    cp_async_wait<0>();
}

template <typename T, int TJ, int NS, bool CS>
size_t pipe_smem() {
    return (size_t)(NS * PipeLayout<TJ, CS>::kStage + 4 * PipeLayout<TJ, CS>::kTile) * sizeof(T);
}

// The pipelined variants: (stages, coefficients staged, min CTAs per SM).
template <typename T, typename F>
bool pipe_dispatch(int variant, F&& f) {
    switch (variant) {
        case 2: f.template run<3, true, 3>(); return true;
        case 3: f.template run<4, true, 2>(); return true;
        case 4: f.template run<3, false, 4>(); return true;
        case 5: f.template run<4, false, 4>(); return true;
        case 6: f.template run<4, false, 3>(); return true;
        default: return false;
    }
}

template <typename T>
struct PipePrepare {
    cudaError_t err = cudaSuccess;
    template <int NS, bool CS, int MINB>
    void run() {
        err = cudaFuncSetAttribute(k_step_fused_pipe<T, 8, NS, CS, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)pipe_smem<T, 8, NS, CS>());
    }
};

template <typename T>
struct PipeOcc {
    int a = 0;
    template <int NS, bool CS, int MINB>
    void run() {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_step_fused_pipe<T, 8, NS, CS, MINB>, 256,
                                                      pipe_smem<T, 8, NS, CS>());
    }
};

template <typename T>
struct PipeLaunch {
    const StencilArgs<T>& a;
    dim3 grid;
    cudaStream_t s;
    template <int NS, bool CS, int MINB>
    void run() {
        k_step_fused_pipe<T, 8, NS, CS, MINB><<<grid, 256, pipe_smem<T, 8, NS, CS>(), s>>>(a);
    }
};

}  // namespace

// Fused-step variants: 0 = register prefetch (TJ 8), 1 = register prefetch
// (TJ 16), 2 / 3 = cp.async pipeline of all arrays (TJ 8, 3 / 4 stages),
// 4 / 5 / 6 = cp.async pipeline of E and H with register-prefetched
// coefficients (3 stages at 4 CTAs per SM, 4 stages at 4 and at 3).
int fused_tj_of(int variant) { return variant == 1 ? 16 : 8; }

template <typename T>
cudaError_t prepare_fused(int variant) {
    PipePrepare<T> f;
    pipe_dispatch<T>(variant, f);
    return f.err;
}
template cudaError_t prepare_fused<float>(int);
template cudaError_t prepare_fused<double>(int);

template <typename T>
int fused_occupancy(int variant) {
    int a = 0;
    PipeOcc<T> f;
    if (pipe_dispatch<T>(variant, f))
        a = f.a;
    else if (variant == 1)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_step_fused<T, 16>, 512, 0);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_step_fused<T, 8>, 256, 0);
    return a < 1 ? 1 : a;
}
template int fused_occupancy<float>(int);
template int fused_occupancy<double>(int);

StreamPlan plan_fused(const Geom& g, int sm_count, int ctas_per_sm, int B, int tj) {
    StreamPlan s{};
    s.block_y = tj;
    s.grid_x = (g.nz + 1 + 30) / 31;
    const int ntj = (g.ny + tj - 1) / (tj - 1);
    s.grid_y = ntj * B;
    const long long tiles = (long long)s.grid_x * s.grid_y;
    const int nplanes = g.nx + 1;
    const int per_wave = sm_count * ctas_per_sm;
    double best = -1.0;
    int best_chunk = nplanes;
    for (int ichunk = nplanes; ichunk >= 8; --ichunk) {
        const int nch = (nplanes + ichunk - 1) / ichunk;
        const double waves = (double)tiles * nch / per_wave;
        const double eff = waves / (double)((long long)(waves + 0.999999));
        // a chunk recomputes one E plane: prefer long chunks, but keep at
        // least two waves of CTAs in flight (the march is latency-bound)
        const double score = eff - 1.0 / ichunk - (waves < 2.0 ? 0.5 : 0.0);
        if (score > best) {
            best = score;
            best_chunk = ichunk;
        }
    }
    s.ichunk = best_chunk;
    s.grid_z = (nplanes + best_chunk - 1) / best_chunk;
    return s;
}

template <typename T>
void launch_fused_step(StencilArgs<T> a, const StreamPlan& sp, int variant, cudaStream_t s) {
    a.ichunk = sp.ichunk;
    const dim3 grid(sp.grid_x, sp.grid_y, sp.grid_z);
    PipeLaunch<T> f{a, grid, s};
    if (pipe_dispatch<T>(variant, f)) return;
    if (variant == 1)
        k_step_fused<T, 16><<<grid, 512, 0, s>>>(a);
    else
        k_step_fused<T, 8><<<grid, 256, 0, s>>>(a);
}
template void launch_fused_step<float>(StencilArgs<float>, const StreamPlan&, int, cudaStream_t);
template void launch_fused_step<double>(StencilArgs<double>, const StreamPlan&, int, cudaStream_t);

template <typename T>
void launch_fix_H(const StencilArgs<T>& a, const int4* cells, int n, cudaStream_t s) {
    if (n <= 0) return;
    const long long work = (long long)n * a.B;
    const int threads = 128;
    const long long want = (work + threads - 1) / threads;
    const int blocks = (int)(want < 148 * 8 ? want : 148 * 8);
    k_fix_H<T><<<blocks, threads, 0, s>>>(a, cells, n);
}
template void launch_fix_H<float>(const StencilArgs<float>&, const int4*, int, cudaStream_t);
template void launch_fix_H<double>(const StencilArgs<double>&, const int4*, int, cudaStream_t);

}  // namespace fitb
