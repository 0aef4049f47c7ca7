// Leapfrog curl updates streamed through shared memory by the bulk-copy
// (TMA) engine.
//
// Same arithmetic as stencil.cu (reference: numba_kernels.py:36-127 and
// cpml.py:343-516); only the data movement differs.  A CTA owns a tile of
// TJ whole rows (all k) of the padded box and marches over a chunk of i
// planes.  In the padded layout a run of whole rows is one contiguous,
// 16-byte-aligned range, so each array of a plane tile arrives with a
// single cp.async.bulk copy issued by one thread and completing on an
// mbarrier.  A ring of S stages keeps S-2 planes in flight while the CTA
// computes plane i from stages i and i-1 (the x-neighbours live in the
// previous stage); all stencil neighbours are read from shared memory.
//
// Stage layout (rows of nkp elements):
//   E kernel: aE(3 x TJ)  bE(3 x TJ)  E(3 x TJ)  H(3 x (TJ+1), from row j0-1)
//   H kernel: aH(3 x TJ)  bH(3 x TJ)  H(3 x TJ)  E(3 x (TJ+1), from row j0)
// The E kernel's first stage (plane i0-1) only carries H; the H kernel's
// last stage (plane i1) only carries E.
//
// Every wait on an mbarrier is bounded; on expiry the CTA records a status
// code, waits (bounded) for its own copies still in flight, and returns.
#include "fitb_common.cuh"

namespace fitb {

namespace {

constexpr unsigned kWaitLimit = 1u << 24;

__device__ __forceinline__ unsigned smem_addr(const void* p) {
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait; false when the limit expired.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity) {
    for (unsigned n = 0; n < kWaitLimit; ++n)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

template <typename T>
__device__ __forceinline__ long long slab_at(const FaceDev& f, int l, int i, int j, int k) {
    const int a = (f.axis == 0) ? l : i;
    const int b = (f.axis == 1) ? l : j;
    const int c = (f.axis == 2) ? l : k;
    return ((long long)a * f.dJ + b) * f.pk + c;
}

// Shared-memory ring bookkeeping common to both kernels.
struct Ring {
    unsigned long long* bars;
    unsigned char* base;
    size_t stage_bytes;
    int S;
};

template <typename T>
__device__ __forceinline__ T* stage_ptr(const Ring& r, int it) {
    return reinterpret_cast<T*>(r.base + (size_t)(it % r.S) * r.stage_bytes);
}

// Called by all threads after a failed wait: agree, drain own copies
// (bounded), report.  Returns true when the CTA must stop.
__device__ bool ring_abort(const Ring& r, bool failed, int n_issued, int it_failed, int* status, int code) {
    const int any = __syncthreads_or(failed ? 1 : 0);
    if (!any) return false;
    if (threadIdx.x == 0) {
        atomicExch(status, code);
        for (int it = it_failed; it < n_issued; ++it) mbar_wait_bounded(&r.bars[it % r.S], (unsigned)((it / r.S) & 1));
    }
    __syncthreads();
    return true;
}

template <typename T, int TJ>
__global__ void __launch_bounds__(512) k_update_E_bulk(const StencilArgs<T> p, const int ichunk, const int S,
                                                       int* status) {
    extern __shared__ __align__(128) unsigned char smem[];
    const Geom& g = p.g;
    const int nkp = g.nkp;
    const long long vol = g.vol;
    const int j0 = blockIdx.x * TJ;
    const int i0 = blockIdx.y * ichunk;
    const int i1 = min(i0 + ichunk, g.nx + 1);
    const int nplanes = (i1 - i0) + 1;  // planes i0-1 .. i1-1
    const size_t row_bytes = (size_t)nkp * sizeof(T);
    Ring r;
    r.bars = reinterpret_cast<unsigned long long*>(smem);
    r.base = smem + 128;
    r.stage_bytes = (size_t)(12 * TJ + 3) * row_bytes;
    r.S = S;
    T* E = p.e;
    const T* H = p.h;
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) mbar_init(&r.bars[s], 1);
        fence_barrier_init();
    }
    __syncthreads();

    auto issue = [&](int it) {
        T* st = stage_ptr<T>(r, it);
        const int i = i0 - 1 + it;
        const unsigned hb = (unsigned)((TJ + 1) * row_bytes);
        const unsigned cb = (unsigned)(TJ * row_bytes);
        unsigned long long* bar = &r.bars[it % S];
        const bool full = it > 0;
        mbar_arrive_expect_tx(bar, 3 * hb + (full ? 9 * cb : 0));
        if (full) {
            for (int c = 0; c < 3; ++c) {
                bulk_g2s(st + (size_t)(c * TJ) * nkp, p.aE + c * vol + pidx(g, i, j0, 0), cb, bar);
                bulk_g2s(st + (size_t)((3 + c) * TJ) * nkp, p.bE + c * vol + pidx(g, i, j0, 0), cb, bar);
                bulk_g2s(st + (size_t)((6 + c) * TJ) * nkp, E + c * vol + pidx(g, i, j0, 0), cb, bar);
            }
        }
        for (int c = 0; c < 3; ++c)
            bulk_g2s(st + (size_t)(9 * TJ + c * (TJ + 1)) * nkp, H + c * vol + pidx(g, i, j0 - 1, 0), hb, bar);
    };

    int n_issued = 0;
    if (threadIdx.x == 0) {
        fence_proxy_async();
        for (; n_issued < min(S, nplanes); ++n_issued) issue(n_issued);
    }
    for (int it = 0; it < nplanes; ++it) {
        const bool ok = mbar_wait_bounded(&r.bars[it % S], (unsigned)((it / S) & 1));
        if (ring_abort(r, !ok, threadIdx.x == 0 ? n_issued : 0, it, status, kStatusWaitTimeoutE)) return;
        if (it >= 1) {
            const int i = i0 - 1 + it;
            const T* cur = stage_ptr<T>(r, it);
            const T* prv = stage_ptr<T>(r, it - 1);
            const T* hx_s = cur + (size_t)(9 * TJ) * nkp;
            const T* hy_s = hx_s + (size_t)(TJ + 1) * nkp;
            const T* hz_s = hy_s + (size_t)(TJ + 1) * nkp;
            const T* hy_p = prv + (size_t)(9 * TJ + (TJ + 1)) * nkp;
            const T* hz_p = hy_p + (size_t)(TJ + 1) * nkp;
            for (int cell = threadIdx.x; cell < TJ * nkp; cell += blockDim.x) {
                const int rr = cell / nkp;
                const int k = cell - rr * nkp;
                const int j = j0 + rr;
                if (j > g.ny || k > g.nz) continue;
                const int q = (rr + 1) * nkp + k;  // H row index of (j, k)
                const T hx = hx_s[q], hy = hy_s[q], hz = hz_s[q];
                const T hx_jm = hx_s[q - nkp], hz_jm = hz_s[q - nkp];
                const T hx_km = hx_s[q - 1], hy_km = hy_s[q - 1];
                const T hy_im = hy_p[q], hz_im = hz_p[q];
                const T cx = ((hz - hz_jm) - hy) + hy_km;
                const T cy = ((hx - hx_km) - hz) + hz_im;
                const T cz = ((hy - hy_im) - hx) + hx_jm;
                const int o = rr * nkp + k;
                const T bex = cur[(size_t)(3 * TJ) * nkp + o];
                const T bey = cur[(size_t)(4 * TJ) * nkp + o];
                const T bez = cur[(size_t)(5 * TJ) * nkp + o];
                T ex = cur[o] * cur[(size_t)(6 * TJ) * nkp + o] + bex * cx;
                T ey = cur[(size_t)TJ * nkp + o] * cur[(size_t)(7 * TJ) * nkp + o] + bey * cy;
                T ez = cur[(size_t)(2 * TJ) * nkp + o] * cur[(size_t)(8 * TJ) * nkp + o] + bez * cz;
                for (int fi = 0; fi < p.nfaces; ++fi) {
                    const FaceDev& f = p.f[fi];
                    const int coord = (f.axis == 0) ? i : ((f.axis == 1) ? j : k);
                    const int l = coord - f.lo;
                    if ((unsigned)l >= (unsigned)f.n) continue;
                    const long long s = slab_at<T>(f, l, i, j, k);
                    const T* bcc = static_cast<const T*>(f.bcc);
                    const T cb = bcc[l], cc = bcc[f.n + l], cck = bcc[2 * f.n + l];
                    T* psi = static_cast<T*>(f.psi);
                    T d1, d2;
                    if (f.axis == 0) {
                        d1 = hz - hz_im;
                        d2 = hy - hy_im;
                    } else if (f.axis == 1) {
                        d1 = hz - hz_jm;
                        d2 = hx - hx_jm;
                    } else {
                        d1 = hy - hy_km;
                        d2 = hx - hx_km;
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
                const long long go = pidx(g, i, j, k);
                E[go] = ex;
                E[vol + go] = ey;
                E[2 * vol + go] = ez;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0 && it >= 1 && n_issued < nplanes) {
            fence_proxy_async();
            issue(n_issued);
            ++n_issued;
        }
    }
}

template <typename T, int TJ>
__global__ void __launch_bounds__(512) k_update_H_bulk(const StencilArgs<T> p, const int ichunk, const int S,
                                                       int* status) {
    extern __shared__ __align__(128) unsigned char smem[];
    const Geom& g = p.g;
    const int nkp = g.nkp;
    const long long vol = g.vol;
    const int j0 = blockIdx.x * TJ;
    const int i0 = blockIdx.y * ichunk;
    const int i1 = min(i0 + ichunk, g.nx + 1);
    const int nplanes = (i1 - i0) + 1;  // planes i0 .. i1
    const size_t row_bytes = (size_t)nkp * sizeof(T);
    Ring r;
    r.bars = reinterpret_cast<unsigned long long*>(smem);
    r.base = smem + 128;
    r.stage_bytes = (size_t)(12 * TJ + 3) * row_bytes;
    r.S = S;
    const T* E = p.e;
    T* H = p.h;
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) mbar_init(&r.bars[s], 1);
        fence_barrier_init();
    }
    __syncthreads();

    auto issue = [&](int it) {
        T* st = stage_ptr<T>(r, it);
        const int i = i0 + it;
        const unsigned eb = (unsigned)((TJ + 1) * row_bytes);
        const unsigned cb = (unsigned)(TJ * row_bytes);
        unsigned long long* bar = &r.bars[it % S];
        const bool full = it < nplanes - 1;
        mbar_arrive_expect_tx(bar, 3 * eb + (full ? 9 * cb : 0));
        if (full) {
            for (int c = 0; c < 3; ++c) {
                bulk_g2s(st + (size_t)(c * TJ) * nkp, p.aH + c * vol + pidx(g, i, j0, 0), cb, bar);
                bulk_g2s(st + (size_t)((3 + c) * TJ) * nkp, p.bH + c * vol + pidx(g, i, j0, 0), cb, bar);
                bulk_g2s(st + (size_t)((6 + c) * TJ) * nkp, H + c * vol + pidx(g, i, j0, 0), cb, bar);
            }
        }
        for (int c = 0; c < 3; ++c)
            bulk_g2s(st + (size_t)(9 * TJ + c * (TJ + 1)) * nkp, E + c * vol + pidx(g, i, j0, 0), eb, bar);
    };

    int n_issued = 0;
    if (threadIdx.x == 0) {
        fence_proxy_async();
        for (; n_issued < min(S, nplanes); ++n_issued) issue(n_issued);
    }
    for (int it = 0; it < nplanes; ++it) {
        const bool ok = mbar_wait_bounded(&r.bars[it % S], (unsigned)((it / S) & 1));
        if (ring_abort(r, !ok, threadIdx.x == 0 ? n_issued : 0, it, status, kStatusWaitTimeoutH)) return;
        if (it >= 1) {
            const int i = i0 + it - 1;
            const T* cur = stage_ptr<T>(r, it - 1);
            const T* nxt = stage_ptr<T>(r, it);
            const T* ex_s = cur + (size_t)(9 * TJ) * nkp;
            const T* ey_s = ex_s + (size_t)(TJ + 1) * nkp;
            const T* ez_s = ey_s + (size_t)(TJ + 1) * nkp;
            const T* ey_n = nxt + (size_t)(9 * TJ + (TJ + 1)) * nkp;
            const T* ez_n = ey_n + (size_t)(TJ + 1) * nkp;
            for (int cell = threadIdx.x; cell < TJ * nkp; cell += blockDim.x) {
                const int rr = cell / nkp;
                const int k = cell - rr * nkp;
                const int j = j0 + rr;
                if (j > g.ny || k > g.nz) continue;
                const int q = rr * nkp + k;
                const T ex = ex_s[q], ey = ey_s[q], ez = ez_s[q];
                const T ez_jp = ez_s[q + nkp], ex_jp = ex_s[q + nkp];
                const T ey_kp = ey_s[q + 1], ex_kp = ex_s[q + 1];
                const T ez_ip = ez_n[q], ey_ip = ey_n[q];
                const T cx = ((ez_jp - ez) - ey_kp) + ey;
                const T cy = ((ex_kp - ex) - ez_ip) + ez;
                const T cz = ((ey_ip - ey) - ex_jp) + ex;
                const T bhx = cur[(size_t)(3 * TJ) * nkp + q];
                const T bhy = cur[(size_t)(4 * TJ) * nkp + q];
                const T bhz = cur[(size_t)(5 * TJ) * nkp + q];
                T hx = cur[q] * cur[(size_t)(6 * TJ) * nkp + q] - bhx * cx;
                T hy = cur[(size_t)TJ * nkp + q] * cur[(size_t)(7 * TJ) * nkp + q] - bhy * cy;
                T hz = cur[(size_t)(2 * TJ) * nkp + q] * cur[(size_t)(8 * TJ) * nkp + q] - bhz * cz;
                for (int fi = 0; fi < p.nfaces; ++fi) {
                    const FaceDev& f = p.f[fi];
                    const int coord = (f.axis == 0) ? i : ((f.axis == 1) ? j : k);
                    const int l = coord - f.lo;
                    if ((unsigned)l >= (unsigned)f.n) continue;
                    const long long s = slab_at<T>(f, l, i, j, k);
                    const T* bcc = static_cast<const T*>(f.bcc);
                    const T cb = bcc[l], cc = bcc[f.n + l], cck = bcc[2 * f.n + l];
                    T* psi = static_cast<T*>(f.psi);
                    T d1, d2;
                    if (f.axis == 0) {
                        d1 = ez_ip - ez;
                        d2 = ey_ip - ey;
                    } else if (f.axis == 1) {
                        d1 = ez_jp - ez;
                        d2 = ex_jp - ex;
                    } else {
                        d1 = ey_kp - ey;
                        d2 = ex_kp - ex;
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
                const long long go = pidx(g, i, j, k);
                H[go] = hx;
                H[vol + go] = hy;
                H[2 * vol + go] = hz;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0 && it >= 1 && n_issued < nplanes) {
            fence_proxy_async();
            issue(n_issued);
            ++n_issued;
        }
    }
}

}  // namespace

template <typename T>
BulkPlan plan_bulk(const Geom& g, int sm_count) {
    BulkPlan b{};
    const size_t row = (size_t)g.nkp * sizeof(T);
    const size_t budget = 112 * 1024 - 128;  // two CTAs per SM when it fits
    b.tj = ((12 * 2 + 3) * row * 4 <= budget) ? 2 : 1;
    const size_t stage = (size_t)(12 * b.tj + 3) * row;
    int S = (int)(budget / stage);
    if (S < 3) S = (int)((227 * 1024 - 128) / stage);  // one CTA per SM
    b.stages = S < 3 ? 0 : (S > 6 ? 6 : S);
    b.smem = 128 + (size_t)b.stages * stage;
    int cells = b.tj * g.nkp;
    int thr = ((cells + 1) / 2 + 31) / 32 * 32;
    b.threads = thr < 128 ? 128 : (thr > 512 ? 512 : thr);
    b.ntiles = (g.ny + 1 + b.tj - 1) / b.tj;
    const int occ = (b.smem * 2 <= 227 * 1024) ? 2 : 1;
    const int per_wave = sm_count * occ;
    const int nplanes = g.nx + 1;
    // chunks along i: at least 8 planes each, best wave efficiency
    double best = -1.0;
    int best_n = 1;
    for (int nch = 1; nch <= nplanes; ++nch) {
        const int ichunk = (nplanes + nch - 1) / nch;
        if (ichunk < 8 && nch > 1) break;
        const int nchunk_real = (nplanes + ichunk - 1) / ichunk;
        const double ctas = (double)b.ntiles * nchunk_real;
        const double waves = ctas / per_wave;
        const double eff = waves / (double)((long long)(waves + 0.999999));
        const double score = eff - 0.01 * (double)(1.0 / ichunk) * 8.0;  // prefer long chunks
        if (score > best + 1e-9) {
            best = score;
            best_n = nchunk_real;
        }
    }
    b.ichunk = (nplanes + best_n - 1) / best_n;
    b.nchunks = (nplanes + b.ichunk - 1) / b.ichunk;
    return b;
}

template <typename T>
void launch_update_E_bulk(const StencilArgs<T>& a, const BulkPlan& plan, int* status, cudaStream_t s) {
    dim3 grid(plan.ntiles, plan.nchunks, 1);
    if (plan.tj == 2)
        k_update_E_bulk<T, 2><<<grid, plan.threads, plan.smem, s>>>(a, plan.ichunk, plan.stages, status);
    else
        k_update_E_bulk<T, 1><<<grid, plan.threads, plan.smem, s>>>(a, plan.ichunk, plan.stages, status);
}

template <typename T>
void launch_update_H_bulk(const StencilArgs<T>& a, const BulkPlan& plan, int* status, cudaStream_t s) {
    dim3 grid(plan.ntiles, plan.nchunks, 1);
    if (plan.tj == 2)
        k_update_H_bulk<T, 2><<<grid, plan.threads, plan.smem, s>>>(a, plan.ichunk, plan.stages, status);
    else
        k_update_H_bulk<T, 1><<<grid, plan.threads, plan.smem, s>>>(a, plan.ichunk, plan.stages, status);
}

template <typename T>
cudaError_t prepare_bulk(const BulkPlan& plan) {
    const int smem = (int)plan.smem;
    cudaError_t e = cudaSuccess;
    for (cudaError_t x : {cudaFuncSetAttribute(k_update_E_bulk<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem),
                          cudaFuncSetAttribute(k_update_E_bulk<T, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem),
                          cudaFuncSetAttribute(k_update_H_bulk<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem),
                          cudaFuncSetAttribute(k_update_H_bulk<T, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)})
        if (x != cudaSuccess) e = x;
    return e;
}

template cudaError_t prepare_bulk<float>(const BulkPlan&);
template cudaError_t prepare_bulk<double>(const BulkPlan&);
template BulkPlan plan_bulk<float>(const Geom&, int);
template BulkPlan plan_bulk<double>(const Geom&, int);
template void launch_update_E_bulk<float>(const StencilArgs<float>&, const BulkPlan&, int*, cudaStream_t);
template void launch_update_E_bulk<double>(const StencilArgs<double>&, const BulkPlan&, int*, cudaStream_t);
template void launch_update_H_bulk<float>(const StencilArgs<float>&, const BulkPlan&, int*, cudaStream_t);
template void launch_update_H_bulk<double>(const StencilArgs<double>&, const BulkPlan&, int*, cudaStream_t);

}  // namespace fitb
